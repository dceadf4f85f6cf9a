"""The FP64 CPU oracle against the reference: golden traces written by the
reference programs, and (where oracle/_ref/ is built) the reference's own
update functions on random states, compared bit for bit."""
import glob
import math
import os

import numpy as np
import pytest

import harness as H
from golden import make_golden as G
from oracle import oracle as O

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith("segy_"))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference_traces(path):
    p, kind, program, ref_t, ref_v = G.load(path)
    if kind == "eiso":
        tr, tt, _ = H.run_eiso_oracle(p)
    elif kind == "ecyl":
        tr, tt, _ = H.run_ecyl_oracle(p)
    else:
        tr, tt, _ = H.run_a3d_oracle(p)
    assert [len(a) for a in tr] == [len(a) for a in ref_v]
    for a, b in zip(tt, ref_t):
        np.testing.assert_allclose(a, b, rtol=1e-6)
    if kind == "ecyl":
        # components differ by orders of magnitude (stresses, velocities,
        # div, curl) and some traces hold only round-off before the wave
        # arrives: compare each component over all of its records
        for comp in sorted({r[0] for r in p.receivers}):
            ks = [k for k, r in enumerate(p.receivers) if r[0] == comp]
            a = np.concatenate([tr[k] for k in ks])
            b = np.concatenate([ref_v[k] for k in ks])
            if np.abs(b).max() == 0.0:
                assert np.abs(a).max() == 0.0, comp
            else:
                assert O.rel_l2(a, b) < 2e-6, comp
        return
    # the reference prints 7 significant digits ("%le"), so agreement is
    # bounded by text precision, not by arithmetic
    for a, b in zip(tr, ref_v):
        assert O.rel_l2(a, b) < 2e-6
    assert H.rel_l2(tr, ref_v) < 1e-6


def _random_state(ref, orc, rng):
    P, nx, nz = ref.np, ref.nx, ref.nz
    NX, NZ = nx + 2 * P, nz + 2 * P
    inter = np.zeros((NX, NZ), bool)
    inter[P:P + nx, P:P + nz] = True
    for f in ("vx", "vz", "txx", "tzz", "txz"):
        tot, xp, zp = (rng.standard_normal((NX, NZ)) for _ in range(3))
        xp[inter] = 0
        zp[inter] = 0
        orc.set(f, "x", xp)
        orc.set(f, "z", zp)
        orc.set(f, "total", np.where(inter, tot, 0))
        ref.f[f][:] = tot[P:P + nx, P:P + nz].reshape(-1)
        ref.s[f + "_x"][:] = O.padded_to_regions(xp, nx, nz, P)
        ref.s[f + "_z"][:] = O.padded_to_regions(zp, nx, nz, P)


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent (oracle/_ref)")
@pytest.mark.parametrize("shape", [(13, 9, 3), (9, 14, 4), (20, 20, 5), (17, 11, 2), (8, 8, 1)])
def test_oracle_bitwise_vs_reference_functions(shape):
    nx, nz, P = shape
    rng = np.random.default_rng(sum(shape))
    vp = 3000 + 500 * rng.random((nx, nz))
    vs = vp / 1.8
    rho = 2000 + 300 * rng.random((nx, nz))
    la, mu, l2m, b, bm, vpmax = O.eiso_materials(vp, vs, rho)
    h = 1.0
    dt = 0.5 * h / (math.sqrt(2) * vpmax)
    d, dh, dH = O.eiso_profiles(P, h, vp)
    # nx > nz: the reference's lower-right corner reads past its arrays
    # (pml.c:1044-1084); compare with the build that reads [nx*nz-1]
    ref = O.RefEIso(nx, nz, P, h, dt, la, mu, l2m, b, bm, d, dh, dH, lrfix=nx > nz)
    orc = O.EIso(nx, nz, P, h, dt, la, mu, l2m, b, bm, d, dh, dH)
    _random_state(ref, orc, rng)
    for _ in range(3):
        ref.velocity()
        orc.velocity()
        ref.stress()
        orc.stress()
    for f in ("vx", "vz", "txx", "tzz", "txz"):
        for part in ("total", "x", "z"):
            np.testing.assert_array_equal(orc.get(f, part), ref.padded(f, part))


def test_ricker_properties():
    dt = 1e-4
    w = O.src_fct([2.5], [50.0], dt)[0]
    assert len(w) == math.ceil(2.0 / (50.0 * dt))
    assert abs(np.abs(w).max() - 2.5) < 1e-12
    # zero-phase Ricker, symmetric about tcut = 1/f
    k = int(round(1.0 / (50.0 * dt)))
    np.testing.assert_allclose(w[k - 5:k], w[k + 5:k:-1], rtol=1e-9)


def test_ricker_multi_source_normalisation():
    # src.c:43-65 rescales wavelet 0 on every pass: its final peak is the
    # last source's A, and later wavelets keep their raw amplitude
    dt = 1e-4
    w = O.src_fct([1.0, 3.0], [50.0, 50.0], dt)
    assert abs(np.abs(w[0]).max() - 3.0) < 1e-12
    raw = 3.0 * 2 * math.pi ** 2 * 50.0 ** 2
    assert abs(np.abs(w[1]).max() - raw) / raw < 1e-3


def test_sampling_predicate_edges():
    dt = 1e-4
    assert H.sample_schedule(10, dt, 0.0, dt) == list(range(10))
    assert H.sample_schedule(10, dt, 0.0, 2 * dt) == [1, 3, 5, 7, 9]
    # rdt <= 0: a single sample at t0
    assert H.sample_schedule(10, dt, 5 * dt, 0.0) == [4]
    assert O.nsteps(1500 * dt, dt) in (1500, 1501)
