"""CPU checks of libseismod_gpu.so: it loads, exports every symbol the public
header declares, its host-side set-up (C, FP64) equals the oracle bit for
bit, and argument errors come back as status codes (no GPU needed)."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import oracle as O
from seismod_b200 import _lib as L
from seismod_b200 import api
from seismod_b200 import workloads as W


def test_library_exports_every_header_symbol():
    lib = L.load()
    syms = L.header_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert lib.sm_abi_version() == 1


def test_ricker_matches_oracle_bitwise():
    for A, f, dt in [([1.0], [50.0], 8.8e-5), ([2.0, 0.5, 1.5], [60.0, 60.0, 40.0], 1e-4),
                     ([1.0], [15.0], 1.7e-4)]:
        fct, ln = api.ricker(A, f, dt)
        ref = O.src_fct(A, f, dt)
        for s in range(len(A)):
            assert ln[s] == len(ref[s])
            np.testing.assert_array_equal(fct[s, :ln[s]], ref[s])


def test_eiso_setup_matches_oracle_bitwise():
    rng = np.random.default_rng(3)
    for nx, nz in [(7, 5), (5, 9), (30, 30)]:
        vp = 2000 + 3000 * rng.random((nx, nz))
        vs = vp / (1.5 + rng.random((nx, nz)))
        rho = 1500 + 1000 * rng.random((nx, nz))
        a = api.eiso_materials(vp, vs, rho)
        b = O.eiso_materials(vp, vs, rho)
        for x, y in zip(a[:5], b[:5]):
            np.testing.assert_array_equal(x, y)
        assert a[5] == b[5]
        for npml in (1, 4, 20):
            for x, y in zip(api.eiso_profiles(npml, 1.5, vp), O.eiso_profiles(npml, 1.5, vp)):
                np.testing.assert_array_equal(x, y)


def test_a3d_setup_matches_oracle_bitwise():
    rng = np.random.default_rng(4)
    vp = 1500 + 3000 * rng.random((6, 7, 8))
    rho = 1800 + 500 * rng.random((6, 7, 8))
    for npml in (1, 3):
        a = api.a3d_pad_model(vp, rho, npml)
        b = O.a3d_pad_model(vp, rho, npml)
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])
        assert api.a3d_cfl_vpmax(6, 8, a[0]) == O.a3d_cfl_vpmax(6, 8, b[0])
        shp = a[0].shape
        for (Rc, km, am, f0) in [(1e-5, 1.0, 1, 25.0), (1e-3, 3.0, 0, 10.0)]:
            x = api.a3d_cpml(npml, shp, (5.0, 4.0, 3.0), 1e-4, 2.0, 5000.0, Rc, km, am, f0)
            y = O.a3d_cpml(npml, shp, 5.0, 4.0, 3.0, 1e-4, 2.0, 5000.0, Rc, km, am, f0)
            for u, v in zip(x, y):
                np.testing.assert_array_equal(u, v)


def test_a3d_pad_model_split_over_threads_equals_the_oracle():
    # above 2^20 padded cells the padding runs on several host threads, each
    # owning a range of x planes: edge planes, rows and columns must come out
    # as the single-threaded oracle pads them
    rng = np.random.default_rng(5)
    for shape, npml in [((61, 70, 83), 16), ((100, 9, 1100), 5), ((3, 400, 900), 1)]:
        vp = 1500 + 3000 * rng.random(shape)
        rho = 1800 + 500 * rng.random(shape)
        a = api.a3d_pad_model(vp, rho, npml)
        b = O.a3d_pad_model(vp, rho, npml)
        assert a[0].size >= 1 << 20
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])


def test_a3d_cfl_vpmax_from_the_unpadded_model_equals_the_padded_scan():
    # the reference scans padded indices i*nz + j (i < nx, j < nz); read
    # from the unpadded model they must land on the nodes padding copies
    # there, including the first planes' padded rows and columns
    rng = np.random.default_rng(6)
    for shape, npml in [((6, 7, 8), 1), ((6, 7, 8), 3), ((40, 3, 50), 16), ((9, 30, 2), 4),
                        ((2, 2, 2), 0)]:
        for trial in range(3):
            vp = 1500 + 3000 * rng.random(shape)
            if trial == 1:   # the maximum on an edge that padding replicates
                vp[0, 0, :] += 5000
            elif trial == 2:
                vp[:, -1, -1] += 5000
            vpp, _ = O.a3d_pad_model(vp, vp, npml)
            nx, _, nz = shape
            assert api.a3d_cfl_vpmax_unpadded(vp, npml) == O.a3d_cfl_vpmax(nx, nz, vpp)


def test_sampling_and_nsteps_match_oracle():
    for dt in (8.838834764831844e-05, 1e-4, 1.7e-4):
        for (t0, rdt) in [(0.0, dt), (0.0, 3 * dt), (2e-3, dt), (5 * dt, 0.0), (0.0, 2.5 * dt)]:
            for it in range(200):
                assert api.sample_predicate(it, dt, t0, rdt) == O.sample(it, dt, t0, rdt)
        for n in (1, 7, 1500, 2000):
            dur = W.steps_duration(n, dt * 1e3)
            assert api.nsteps(dur, dt * 1e3 * 1e-3) == O.nsteps(dur, dt * 1e3 * 1e-3) == n


def test_argument_errors_are_status_codes():
    lib = L.load()
    h = C.c_void_p()
    z = np.zeros(4)
    # nx < 2
    rc = lib.sm_eiso_create(0, 1, 5, 2, 1.0, 1e-4, *[L.dptr(z)] * 8, 0, 1, C.byref(h))
    assert rc == L.SM_EINVAL and b"nx" in lib.sm_last_error()
    # npml = 0: the reference indexes [npml-1]
    rc = lib.sm_eiso_create(0, 5, 5, 0, 1.0, 1e-4, *[L.dptr(z)] * 8, 0, 1, C.byref(h))
    assert rc == L.SM_EINVAL and b"npml" in lib.sm_last_error()
    # unknown precision
    rc = lib.sm_eiso_create(0, 5, 5, 2, 1.0, 1e-4, *[L.dptr(z)] * 8, 9, 1, C.byref(h))
    assert rc == L.SM_EINVAL
    # NULL handle
    assert lib.sm_eiso_run(None, 1) == L.SM_EINVAL
    assert lib.sm_a3d_run(None, 1) == L.SM_EINVAL
    assert lib.sm_eiso_destroy(None) == L.SM_OK
    # ricker with a stride shorter than the wavelet
    fct = np.zeros(4)
    ln = np.zeros(1, dtype=np.uintp)
    A = np.array([1.0])
    f = np.array([50.0])
    rc = lib.sm_ricker(1, L.dptr(A), L.dptr(f), 1e-4, 1.0, 4, L.dptr(fct), L.szptr(ln))
    assert rc == L.SM_EINVAL
    # the unpadded a_iso_3d create: an empty model, a NULL array, no handle
    # pointer (all refused before any device is touched)
    cf = (L._dp * 18)(*[L.dptr(z)] * 18)
    rc = lib.sm_a3d_create_unpadded(0, 0, 4, 4, 1, 1.0, 1.0, 1.0, 1e-4, L.dptr(z), L.dptr(z),
                                    cf, 0, C.byref(h))
    assert rc == L.SM_EINVAL and b"empty" in lib.sm_last_error()
    rc = lib.sm_a3d_create_unpadded(0, 4, 4, 4, 1, 1.0, 1.0, 1.0, 1e-4, None, L.dptr(z),
                                    cf, 0, C.byref(h))
    assert rc == L.SM_EINVAL and b"NULL" in lib.sm_last_error()
    rc = lib.sm_a3d_create_unpadded(0, 4, 4, 4, 1, 1.0, 1.0, 1.0, 1e-4, L.dptr(z), L.dptr(z),
                                    cf, 0, None)
    assert rc == L.SM_EINVAL


def test_a3d_rejects_coefficients_that_are_not_reference_defaults_inside():
    lib = L.load()
    shp = (10, 10, 10)
    coef = api.a3d_cpml(2, shp, (5.0, 5.0, 5.0), 1e-4, f0=10.0)
    coef[0][5] = 0.1  # a != 0 inside the frame
    P = (L._dp * 18)(*[L.dptr(c) for c in coef])
    vp = np.full(shp, 2000.0)
    h = C.c_void_p()
    rc = lib.sm_a3d_create(0, 10, 10, 10, 2, 5.0, 5.0, 5.0, 1e-4, L.dptr(vp), L.dptr(vp), P, 0,
                           C.byref(h))
    assert rc == L.SM_EINVAL


def test_c_round_is_half_away_from_zero():
    assert api.c_round(2.5) == 3 and api.c_round(-2.5) == -3 and api.c_round(1.4999) == 1
    assert math.floor(0.5 + 0.5) == api.c_round(0.5)


def test_server_request_structs_match_the_c_layout():
    from seismod_b200 import serving
    e, a, s = serving.struct_sizes()
    assert e == C.sizeof(serving.EisoRequest)
    assert a == C.sizeof(serving.A3dRequest)
    assert s == C.sizeof(serving.ServerStats)


def test_device_bytes_estimates_grow_with_the_problem():
    from seismod_b200 import serving
    lib = serving.lib()
    b1, b2 = C.c_size_t(), C.c_size_t()
    assert lib.sm_eiso_device_bytes(400, 400, 20, 0, 1, 64, 1500, C.byref(b1)) == 0
    assert lib.sm_eiso_device_bytes(400, 400, 20, 0, 64, 64, 1500, C.byref(b2)) == 0
    # two buffer sets of five FP32 fields per shot at least
    assert b2.value > b1.value >= 2 * 5 * 440 * 448 * 4
    assert lib.sm_a3d_device_bytes(288, 288, 288, 16, 2, 0, 0, C.byref(b1)) == 0
    assert lib.sm_a3d_device_bytes(288, 288, 288, 16, 0, 0, 0, C.byref(b2)) == 0
    assert b2.value > b1.value >= 8 * 288 * 288 * 288 * 2
    assert lib.sm_eiso_device_bytes(10, 10, 2, 9, 1, 0, 0, C.byref(b1)) == 1   # bad precision


def test_ecyl_host_setup_equals_the_oracle_bit_for_bit():
    """Materials, CPML coefficients and the Kurkjian wavelet of the library's
    C host code against the oracle's restatement, with and without the
    absorbing layer."""
    from oracle import oracle as O
    import harness as H
    from seismod_b200 import api
    from seismod_b200 import workloads as W
    for kw in (dict(n=1, src="Kurkjian"), dict(n=0, src="Fz", absorb=0),
               dict(n=2, src="Bulk", dx=1.5, dz=1.0)):
        p = W.ecyl_case(nx=34, nz=41, npml=6, nsteps=40, **kw)
        q = api.ecyl_inputs(p)
        s = H.ecyl_setup(p)
        for k, nm in enumerate(O.ECYL_MATS):
            np.testing.assert_array_equal(q["mats"][k], s["mats"][nm], err_msg=nm)
        for k in range(15):
            np.testing.assert_array_equal(q["coef"][k], s["coef"][k])
        srcs = H.ecyl_sources(p, s)
        for k, (idx, typ, w) in enumerate(srcs):
            assert q["src"][0][k] == idx
            np.testing.assert_array_equal(q["src"][2][k][:q["src"][3][k]], w)
        assert q["nsteps"] == s["nsteps"]
