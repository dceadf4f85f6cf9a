/*
 * sm_io.c -- readers of the reference's input files and its trace writer.
 *
 * Formats and semantics follow io_utils.c (cited per function); where the
 * reference would read past a buffer or dereference NULL on a malformed
 * file, these return SM_EIO with a message instead.
 */
#define _GNU_SOURCE
#include "sm_io.h"

#include <ctype.h>
#include <errno.h>
#include <getopt.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/types.h>
#include <stdint.h>
#include <time.h>

void sm_params_defaults(sm_params *p)
{
    /* io_utils.c:63-98 / 100-135 (the fields the two programs read) */
    memset(p, 0, sizeof *p);
    p->dt = 1.e-4;
    p->duration = 1.2;
    strcpy(p->basename, "run01");
    p->iwipe = 0;
    p->np = 20;
    p->segy = 0;
    p->shotpt_no = 1;
    p->simulate_cmp = 0;
    p->plot_strips = 0;
    p->azimuthal_mode = 0;
    p->Rc = 1.e-5;
    p->kappa_max = 1.;
    p->alpha_max = 1;
    p->vmax = 5000.0;
    p->pml_order = 2.;
    p->precision = SM_FP32;
}

static int parse_precision(const char *s, int *out)
{
    if (!strcmp(s, "fp32")) *out = SM_FP32;
    else if (!strcmp(s, "fp64")) *out = SM_FP64;
    else if (!strcmp(s, "fp16")) *out = SM_FP16;
    else if (!strcmp(s, "bf16")) *out = SM_BF16;
    else if (!strcmp(s, "bfp16")) *out = SM_BFP16;
    else return 0;
    return 1;
}

int sm_parse_args(int argc, char **argv, sm_params *p, const char *prog)
{
    /* io_utils.c:156-202: -p file.par, -v (repeatable), -h; -c (checkpoint
     * restart) belongs to the PSTD programs and is refused here */
    const char *par = NULL;
    int c;
    optind = 1;
    while ((c = getopt(argc, argv, "c:hp:vP:")) != -1) {
        switch (c) {
        case 'p': par = optarg; break;
        case 'v': p->verbose++; break;
        case 'P':
            if (!parse_precision(optarg, &p->precision))
                return sm_fail(SM_EINVAL, "%s: -P takes fp32, fp64, fp16 or bf16", prog);
            break;
        case 'c':
            return sm_fail(SM_EINVAL, "%s: checkpoint restart (-c) is not part of this program", prog);
        case 'h':
            return sm_fail(SM_EINVAL, "usage: %s [-v] [-h] [-P fp32|fp64|fp16|bf16] -p parameter_file",
                           prog);
        default:
            return sm_fail(SM_EINVAL, "usage: %s [-v] [-h] [-P fp32|fp64|fp16|bf16] -p parameter_file",
                           prog);
        }
    }
    if (!par) return sm_fail(SM_EINVAL, "usage: %s [-v] [-h] -p parameter_file", prog);
    return sm_read_par(par, p);
}

int sm_read_par(const char *path, sm_params *p)
{
    /* io_utils.c:204-294: "value  # keyword, comment" per line */
    FILE *fid = fopen(path, "r");
    if (!fid) return sm_fail(SM_EIO, "cannot open parameter file %s for reading", path);
    char line[512], value[256], keyword[256];
    int lineno = 0;
    while (fgets(line, sizeof line, fid)) {
        ++lineno;
        if (sscanf(line, "%255s", value) <= 0) continue;
        char *s1 = strchr(line, '#');
        char *s2 = strchr(line, ',');
        if (!s1 || !s2 || s2 < s1) {
            fclose(fid);
            return sm_fail(SM_EIO, "%s:%d: expected \"value  # keyword, comment\"", path, lineno);
        }
        *s2 = '\0';
        if (sscanf(s1 + 1, "%255s", keyword) != 1) continue;
        if (!strcmp(keyword, "model")) snprintf(p->modelfile, sizeof p->modelfile, "%s", value);
        else if (!strcmp(keyword, "source")) snprintf(p->sourcefile, sizeof p->sourcefile, "%s", value);
        else if (!strcmp(keyword, "output")) snprintf(p->outputfile, sizeof p->outputfile, "%s", value);
        else if (!strcmp(keyword, "basename")) snprintf(p->basename, sizeof p->basename, "%s", value);
        else if (!strcmp(keyword, "time")) p->duration = strtod(value, NULL);
        else if (!strcmp(keyword, "dt")) p->dt = strtod(value, NULL) * 0.001;  /* ms -> s */
        else if (!strcmp(keyword, "abs")) p->iwipe = (short)atoi(value);
        else if (!strcmp(keyword, "nl")) p->np = (size_t)atoi(value);
        else if (!strcmp(keyword, "segy")) p->segy = (short)atoi(value);
        else if (!strcmp(keyword, "plstr")) p->plot_strips = atoi(value);
        else if (!strcmp(keyword, "shotpoint")) p->shotpt_no = atoi(value);
        else if (!strcmp(keyword, "simulateCMP")) p->simulate_cmp = atoi(value);
        else if (!strcmp(keyword, "Rc")) p->Rc = strtod(value, NULL);
        else if (!strcmp(keyword, "kappa_max")) p->kappa_max = strtod(value, NULL);
        else if (!strcmp(keyword, "alpha_max")) p->alpha_max = (short)atoi(value);
        else if (!strcmp(keyword, "azimuthal_mode")) p->azimuthal_mode = atoi(value);
        /* check_model, chkpt_inc, pml_median, saveEnergy, EnergyROI:
         * accepted, unused by these programs */
    }
    fclose(fid);
    if (p->iwipe == 0) p->np = 0;   /* io_utils.c:293 */
    return SM_OK;
}

/* Binary model files (no counterpart in the reference, whose ASCII models
 * take minutes to parse at 512^3): the 8 bytes "SEISMODB", then uint32
 * version (1), ndim (2 or 3), nfields (3: vp vs rho for e_iso, 2: vp rho for
 * a_iso_3d), reserved (0); uint64 nx ny nz (ny = 1 in 2-D); float64 dx dy dz
 * x0 y0 z0; then each field's nx*ny*nz float64 values in the ASCII files'
 * order (index (i*ny + j)*nz + k).  All in the host's byte order. */
static const char kModelMagic[8] = {'S', 'E', 'I', 'S', 'M', 'O', 'D', 'B'};

static int model_is_binary(const char *path)
{
    FILE *f = fopen(path, "rb");
    if (!f) return 0;
    char m[8];
    const int yes = fread(m, 1, 8, f) == 8 && memcmp(m, kModelMagic, 8) == 0;
    fclose(f);
    return yes;
}

static int read_model_bin(const char *path, unsigned ndim, unsigned nfields, sm_grid *g,
                          double **out)
{
    FILE *f = fopen(path, "rb");
    if (!f) return sm_fail(SM_EIO, "cannot open %s for reading", path);
    char m[8];
    uint32_t hdr[4];
    uint64_t n[3];
    double d[6];
    if (fread(m, 1, 8, f) != 8 || fread(hdr, 4, 4, f) != 4 || fread(n, 8, 3, f) != 3 ||
        fread(d, 8, 6, f) != 6) {
        fclose(f);
        return sm_fail(SM_EIO, "%s: short binary model header", path);
    }
    if (hdr[0] != 1 || hdr[1] != ndim || hdr[2] != nfields) {
        fclose(f);
        return sm_fail(SM_EIO, "%s: binary model version %u, %u-D, %u fields; expected 1, %u-D, %u",
                       path, hdr[0], hdr[1], hdr[2], ndim, nfields);
    }
    memset(g, 0, sizeof *g);
    g->nx = n[0]; g->ny = n[1]; g->nz = n[2];
    g->dx = d[0]; g->dy = d[1]; g->dz = d[2];
    g->x0 = d[3]; g->y0 = d[4]; g->z0 = d[5];
    if (!g->nx || !g->ny || !g->nz || (ndim == 2 && g->ny != 1)) {
        fclose(f);
        return sm_fail(SM_EIO, "%s: bad binary model dimensions", path);
    }
    const size_t cells = g->nx * g->ny * g->nz;
    for (unsigned k = 0; k < nfields; ++k) out[k] = NULL;
    for (unsigned k = 0; k < nfields; ++k) {
        out[k] = malloc(cells * sizeof(double));
        if (!out[k] || fread(out[k], sizeof(double), cells, f) != cells) {
            for (unsigned j = 0; j <= k; ++j) { free(out[j]); out[j] = NULL; }
            fclose(f);
            return sm_fail(SM_EIO, "%s: binary model data too short", path);
        }
    }
    fclose(f);
    return SM_OK;
}

/* the values of a text model, on host threads (below) */
static int read_values(FILE *fid, size_t ncol, size_t n, int nf, double *const *v, size_t tnx,
                       size_t tnz, int *is1d);

int sm_read_model_ecyl(const char *path, sm_grid *g, double **pvp, double **pvs, double **prho)
{
    if (model_is_binary(path)) return sm_read_model_e(path, g, pvp, pvs, prho);
    /* io_utils.c:296-328 (grid) and 949-991 (values): the rows are z, r fast
     * within each; a file holding only the first row is a radial profile
     * copied down every row */
    FILE *fid = fopen(path, "r");
    if (!fid) return sm_fail(SM_EIO, "cannot open %s for reading", path);
    char type[64];
    memset(g, 0, sizeof *g);
    g->ny = 1;
    g->dy = 1.0;
    if (fscanf(fid, "%zu %zu", &g->nx, &g->nz) != 2 || fscanf(fid, "%lf %lf", &g->dx, &g->dz) != 2 ||
        fscanf(fid, "%lf %lf", &g->x0, &g->z0) != 2 || fscanf(fid, "%63s", type) != 1) {
        fclose(fid);
        return sm_fail(SM_EIO, "%s: bad header", path);
    }
    if (strcmp(type, "isotropic_elastic_cyl") != 0) {
        fclose(fid);
        return sm_fail(SM_EIO, "model in %s not isotropic_elastic_cyl", path);
    }
    const size_t nx = g->nx, nz = g->nz;
    if (nx < 2 || nz < 2) {
        fclose(fid);
        return sm_fail(SM_EIO, "%s: grid must be at least 2 x 2", path);
    }
    double *vp = malloc(nx * nz * sizeof(double)), *vs = malloc(nx * nz * sizeof(double));
    double *rho = malloc(nx * nz * sizeof(double));
    if (!vp || !vs || !rho) {
        free(vp); free(vs); free(rho); fclose(fid);
        return sm_fail(SM_ENOMEM, "out of host memory");
    }
    int profile = 0;
    double *const va[3] = {vp, vs, rho};
    if (read_values(fid, nx, nx * nz, 3, va, nx, nz, &profile)) {
        fclose(fid); free(vp); free(vs); free(rho);
        return sm_fail(SM_EIO, "something wrong with file %s", path);
    }
    fclose(fid);
    if (profile)
        for (size_t i = 0; i < nx; ++i)
            for (size_t j = 1; j < nz; ++j) {
                vp[i * nz + j] = vp[i * nz];
                vs[i * nz + j] = vs[i * nz];
                rho[i * nz + j] = rho[i * nz];
            }
    *pvp = vp; *pvs = vs; *prho = rho;
    return SM_OK;
}

int sm_read_model_e(const char *path, sm_grid *g, double **pvp, double **pvs, double **prho)
{
    if (model_is_binary(path)) {
        double *a[3];
        int rc = read_model_bin(path, 2, 3, g, a);
        if (rc) return rc;
        if (g->nx < 2 || g->nz < 2) {
            free(a[0]); free(a[1]); free(a[2]);
            return sm_fail(SM_EIO, "%s: grid must be at least 2 x 2", path);
        }
        g->dy = 1.0;
        *pvp = a[0]; *pvs = a[1]; *prho = a[2];
        return SM_OK;
    }
    /* io_utils.c:296-328 (grid) and 892-947 (values; one column = 1-D profile) */
    FILE *fid = fopen(path, "r");
    if (!fid) return sm_fail(SM_EIO, "cannot open %s for reading", path);
    char type[64];
    memset(g, 0, sizeof *g);
    g->ny = 1;
    g->dy = 1.0;
    if (fscanf(fid, "%zu %zu", &g->nx, &g->nz) != 2 || fscanf(fid, "%lf %lf", &g->dx, &g->dz) != 2 ||
        fscanf(fid, "%lf %lf", &g->x0, &g->z0) != 2 || fscanf(fid, "%63s", type) != 1) {
        fclose(fid);
        return sm_fail(SM_EIO, "%s: bad header", path);
    }
    if (strcmp(type, "isotropic_elastic") != 0) {
        fclose(fid);
        return sm_fail(SM_EIO, "model in %s not isotropic_elastic", path);
    }
    const size_t nx = g->nx, nz = g->nz;
    if (nx < 2 || nz < 2) {
        fclose(fid);
        return sm_fail(SM_EIO, "%s: grid must be at least 2 x 2", path);
    }
    double *vp = malloc(nx * nz * sizeof(double)), *vs = malloc(nx * nz * sizeof(double));
    double *rho = malloc(nx * nz * sizeof(double));
    if (!vp || !vs || !rho) {
        free(vp); free(vs); free(rho); fclose(fid);
        return sm_fail(SM_ENOMEM, "out of host memory");
    }
    int flag1d = 0;
    double *const va[3] = {vp, vs, rho};
    if (read_values(fid, nz, nx * nz, 3, va, 0, 0, &flag1d)) goto bad;
    fclose(fid);
    if (flag1d)
        for (size_t i = 1; i < nx; ++i)
            for (size_t j = 0; j < nz; ++j) {
                vp[i * nz + j] = vp[j];
                vs[i * nz + j] = vs[j];
                rho[i * nz + j] = rho[j];
            }
    *pvp = vp; *pvs = vs; *prho = rho;
    return SM_OK;
bad:
    fclose(fid);
    free(vp); free(vs); free(rho);
    return sm_fail(SM_EIO, "something wrong with file %s", path);
}

/* ---------------------------------------------------------------------------
 * Whitespace-separated numbers of a text model, parsed on host threads.  The
 * reference reads one value per fscanf("%lf") call (io_utils.c:1068-1094),
 * minutes for a 512^3 model.  Here the rest of the file is read into memory
 * and cut into chunks at whitespace; pass 1 counts each chunk's tokens, pass 2
 * converts each token with strtod (the conversion fscanf's %lf makes, so the
 * values are the same bits) into its place: token t is field t % nf of the
 * file's cell t / nf, stored at that cell's index (the file's order, or for
 * the cylindrical models, whose rows are z, the transposed one).
 * ------------------------------------------------------------------------- */
typedef struct {
    const char *b, *e;   /* [b, e): starts and ends on a token boundary */
    size_t ntok;         /* pass 1: tokens in the chunk */
    size_t first, need;  /* pass 2: index of the chunk's first token; tokens to convert */
    int nf;              /* fields per cell */
    size_t tnx, tnz;     /* tnx > 0: file cell c is stored at (c % tnx) * tnz + c / tnx */
    double *v[3];        /* field f of the cell -> v[f][cell] */
    size_t bad;          /* first token that is not a whole number, or (size_t)-1 */
} num_chunk;

static void *num_count(void *arg)
{
    num_chunk *c = (num_chunk *)arg;
    size_t n = 0;
    int in = 0;
    for (const char *p = c->b; p < c->e; ++p) {
        const int sp = isspace((unsigned char)*p);
        if (!sp && !in) ++n;
        in = !sp;
    }
    c->ntok = n;
    return NULL;
}

static void *num_convert(void *arg)
{
    num_chunk *c = (num_chunk *)arg;
    size_t t = c->first;
    const char *p = c->b;
    c->bad = (size_t)-1;
    while (p < c->e && t < c->need) {
        while (p < c->e && isspace((unsigned char)*p)) ++p;
        if (p >= c->e) break;
        const char *q = p;
        while (q < c->e && !isspace((unsigned char)*q)) ++q;
        char *end;
        const double x = strtod(p, &end);   /* stops at the whitespace after the token */
        if (end != q) {
            c->bad = t;
            return NULL;
        }
        const size_t cell = t / (size_t)c->nf;
        const size_t at = c->tnx ? (cell % c->tnx) * c->tnz + cell / c->tnx : cell;
        c->v[t % (size_t)c->nf][at] = x;
        ++t;
        p = q;
    }
    return NULL;
}

/* The values after a model header, nf per cell: ncol cells (the first
 * column or row: the profile shortcut) when no number follows them, else all
 * n cells.  *is1d tells which.  Returns 0, or -1 when the file holds fewer
 * numbers than needed or a token that is not a number where one is needed
 * (the reference's "something wrong" cases). */
static int read_values(FILE *fid, size_t ncol, size_t n, int nf, double *const *v, size_t tnx,
                       size_t tnz, int *is1d)
{
    const size_t nfz = (size_t)nf;
    /* the rest of the file, to its end: the buffer is sized from the file's
     * size and grows if more comes (a file still being written) */
    struct stat st;
    const long off = ftell(fid);
    size_t cap = (size_t)1 << 20;
    if (off >= 0 && fstat(fileno(fid), &st) == 0 && S_ISREG(st.st_mode) &&
        (long long)st.st_size >= off)
        cap = (size_t)st.st_size - (size_t)off + 2;   /* + a byte to meet the end, + NUL */
    char *buf = malloc(cap);
    if (!buf) return -1;
    size_t len = 0;
    for (;;) {
        len += fread(buf + len, 1, cap - 1 - len, fid);
        if (len < cap - 1 || feof(fid)) break;
        char *nb = realloc(buf, 2 * cap);   /* full: the input goes on */
        if (!nb) {
            free(buf);
            return -1;
        }
        buf = nb;
        cap *= 2;
    }
    buf[len] = 0;
    const size_t nc = sm_host_threads(len, (size_t)1 << 20);
    num_chunk c[SM_MAX_HOST_THREADS];
    const char *start = buf;
    for (size_t k = 0; k < nc; ++k) {
        const char *e = k + 1 == nc ? buf + len : buf + len * (k + 1) / nc;
        if (e < start) e = start;
        while (e < buf + len && !isspace((unsigned char)*e)) ++e;   /* end at whitespace */
        c[k].b = start;
        c[k].e = e;
        start = e;
    }
    sm_parallel(num_count, c, sizeof c[0], nc);
    size_t ntok = 0;
    for (size_t k = 0; k < nc; ++k) {
        c[k].first = ntok;
        ntok += c[k].ntok;
    }
    int rc = -1;
    if (ntok < nfz * ncol) goto done;
    /* the read of the second column (row) returning nothing -- end of file,
     * or no number at all -- means a profile (io_utils.c:918-946, 970-990,
     * 1074-1080) */
    *is1d = 1;
    if (ntok > nfz * ncol) {
        size_t t = 0, k = 0;   /* the token at index nf*ncol */
        while (k < nc && t + c[k].ntok <= nfz * ncol) t += c[k++].ntok;
        const char *p = c[k].b;
        for (;;) {
            while (isspace((unsigned char)*p)) ++p;
            if (t == nfz * ncol) break;
            while (*p && !isspace((unsigned char)*p)) ++p;
            ++t;
        }
        char *end;
        (void)strtod(p, &end);
        if (end != p) *is1d = 0;
    }
    const size_t need = *is1d ? nfz * ncol : nfz * n;
    if (ntok < need) goto done;
    for (size_t k = 0; k < nc; ++k) {
        c[k].need = need;
        c[k].nf = nf;
        c[k].tnx = tnx;
        c[k].tnz = tnz;
        for (int fl = 0; fl < 3; ++fl) c[k].v[fl] = fl < nf ? v[fl] : NULL;
    }
    sm_parallel(num_convert, c, sizeof c[0], nc);
    rc = 0;
    for (size_t k = 0; k < nc; ++k)
        if (c[k].bad != (size_t)-1) rc = -1;
done:
    free(buf);
    return rc;
}

int sm_read_model_a(const char *path, sm_grid *g, double **pvp, double **prho)
{
    if (model_is_binary(path)) {
        double *a[2];
        int rc = read_model_bin(path, 3, 2, g, a);
        if (rc) return rc;
        *pvp = a[0]; *prho = a[1];
        return SM_OK;
    }
    /* io_utils.c:384-401 (grid) and 1029-1094 (values; one (x,y) column is
     * a 1-D profile).  Returns the nx*ny*nz interior. */
    FILE *fid = fopen(path, "r");
    if (!fid) return sm_fail(SM_EIO, "cannot open %s for reading", path);
    char type[64];
    memset(g, 0, sizeof *g);
    if (fscanf(fid, "%zu %zu %zu", &g->nx, &g->ny, &g->nz) != 3 ||
        fscanf(fid, "%lf %lf %lf", &g->dx, &g->dy, &g->dz) != 3 ||
        fscanf(fid, "%lf %lf %lf", &g->x0, &g->y0, &g->z0) != 3 || fscanf(fid, "%63s", type) != 1) {
        fclose(fid);
        return sm_fail(SM_EIO, "%s: bad header", path);
    }
    if (strcmp(type, "isotropic_acoustic_3d") != 0) {
        fclose(fid);
        return sm_fail(SM_EIO, "model in %s not isotropic_acoustic_3d", path);
    }
    const size_t nx = g->nx, ny = g->ny, nz = g->nz, n = nx * ny * nz;
    if (!nx || !ny || !nz) {
        fclose(fid);
        return sm_fail(SM_EIO, "%s: empty grid", path);
    }
    double *vp = malloc(n * sizeof(double)), *rho = malloc(n * sizeof(double));
    if (!vp || !rho) {
        free(vp); free(rho); fclose(fid);
        return sm_fail(SM_ENOMEM, "out of host memory");
    }
    int flag1d = 0;
    double *const va[2] = {vp, rho};
    if (read_values(fid, nz, n, 2, va, 0, 0, &flag1d)) goto bad;
    fclose(fid);
    if (flag1d)
        for (size_t q = nz; q < n; ++q) {
            vp[q] = vp[q % nz];
            rho[q] = rho[q % nz];
        }
    *pvp = vp; *prho = rho;
    return SM_OK;
bad:
    fclose(fid);
    free(vp); free(rho);
    return sm_fail(SM_EIO, "something wrong with file %s", path);
}

static int source_type(const char *t, int three_d)
{
    /* io_utils.c:1452-1481 (2-D) and 1561-1575 (3-D) */
    char s[64];
    snprintf(s, sizeof s, "%s", t);
    struct { const char *a, *b, *c; int v; int in3d; } tab[] = {
        {"sx", "SX", "Sx", 0, 1}, {"sz", "SZ", "Sz", 2, 1}, {"sxy", "SXY", "Sxy", 3, 0},
        {"sxz", "SXZ", "Sxz", 4, 1}, {"srz", "SRZ", "Srz", 4, 0}, {"syz", "SYZ", "Syz", 5, 0},
        {"sf", "SF", "Sf", 7, 1}, {"bulk", "BULK", "Bulk", 6, 1}, {"bulk_s", "BULK_S", "Bulk_s", 8, 0},
        {"fr", "FR", "Fr", 9, 0}, {"fz", "FZ", "Fz", 11, 0}, {"ftheta", "FTHETA", "Ftheta", 10, 0},
        {"kurkjian", "Kurkjian", "Kurkjian", 12, 0},
    };
    for (size_t q = 0; q < sizeof tab / sizeof tab[0]; ++q)
        if ((!three_d || tab[q].in3d) &&
            (!strcmp(s, tab[q].a) || !strcmp(s, tab[q].b) || !strcmp(s, tab[q].c)))
            return tab[q].v;
    return -1;
}

static long c_round(double v) { return lround(v); }

int sm_read_sources(const char *path, const sm_grid *g, int three_d, sm_source **out,
                    size_t *nout, size_t *ntemplate)
{
    /* io_utils.c:1432-1538 (2-D, 1- or 9-point template) and 1540-1589 (3-D) */
    FILE *fid = fopen(path, "r");
    if (!fid) return sm_fail(SM_EIO, "cannot open %s for reading", path);
    size_t nsrc = 0, ntpl = 1;
    if (fscanf(fid, "%zu", &nsrc) != 1 || nsrc == 0) {
        fclose(fid);
        return sm_fail(SM_EIO, "%s: bad source count", path);
    }
    if (fscanf(fid, "%zu", &ntpl) != 1) ntpl = 1;
    if (three_d && ntpl != 1) {
        fprintf(stdout, "Warning, source template parameter ignored.\n");
        ntpl = 1;
    }
    if (ntpl != 1 && ntpl != 9) {
        fclose(fid);
        return sm_fail(SM_EIO, "%s: template must have 1 or 9 points", path);
    }
    sm_source *s = calloc(nsrc * ntpl, sizeof *s);
    if (!s) { fclose(fid); return sm_fail(SM_ENOMEM, "out of host memory"); }
    char t[64];
    for (size_t n = 0; n < nsrc * ntpl; n += ntpl) {
        if (fscanf(fid, "%63s", t) != 1) goto bad;
        int ty = source_type(t, three_d);
        if (ty < 0) {
            fclose(fid); free(s);
            return sm_fail(SM_EIO, "type of source (%s) not implemented", t);
        }
        s[n].type = ty;
        if (fscanf(fid, "%lf", &s[n].A) != 1 || fscanf(fid, "%lf", &s[n].f) != 1) goto bad;
        if (three_d) {
            if (fscanf(fid, "%lf %lf %lf", &s[n].x, &s[n].y, &s[n].z) != 3) goto bad;
        } else if (fscanf(fid, "%lf %lf", &s[n].x, &s[n].z) != 2) goto bad;
        s[n].i = c_round((s[n].x - g->x0) / g->dx);
        s[n].j = three_d ? c_round((s[n].y - g->y0) / g->dy) : 0;
        s[n].k = c_round((s[n].z - g->z0) / g->dz);
        if (ntpl == 9) {
            /* io_utils.c:1494-1535: centre 1/2, edges 1/4, corners 1/8 */
            const double A = s[n].A;
            static const double w[9] = {0.5, 0.125, 0.25, 0.125, 0.25, 0.25, 0.125, 0.25, 0.125};
            static const int di[9] = {0, -1, 0, 1, -1, 1, -1, 0, 1};
            static const int dk[9] = {0, -1, -1, -1, 0, 0, 1, 1, 1};
            for (int q = 0; q < 9; ++q) {
                s[n + q].type = s[n].type;
                s[n + q].f = s[n].f;
                s[n + q].x = s[n].x;
                s[n + q].z = s[n].z;
                s[n + q].A = w[q] * A;
                s[n + q].i = c_round((s[n].x - g->x0 + di[q] * g->dx) / g->dx);
                s[n + q].k = c_round((s[n].z - g->z0 + dk[q] * g->dz) / g->dz);
            }
        }
    }
    fclose(fid);
    *out = s;
    *nout = nsrc * ntpl;
    *ntemplate = ntpl;
    return SM_OK;
bad:
    fclose(fid);
    free(s);
    return sm_fail(SM_EIO, "something wrong with file %s", path);
}

static int record_comp(const char *t, int three_d)
{
    /* io_utils.c:1607-1649 (2-D) and 1699-1711 (3-D) */
    struct { const char *a, *b, *c; int v; int in3d; } tab[] = {
        {"Vx", "vx", "VX", 0, 1}, {"Vy", "vy", "VY", 1, 1}, {"Vz", "vz", "VZ", 2, 1},
        {"Qx", "qx", "QX", 3, 0}, {"Qz", "qz", "QZ", 4, 0}, {"txx", "TXX", "TXX", 5, 0},
        {"tzz", "TZZ", "TZZ", 6, 0}, {"txy", "TXY", "TXY", 9, 0}, {"tyz", "TYZ", "TYZ", 10, 0},
        {"txz", "TXZ", "TXZ", 7, 0}, {"p", "P", "P", 8, 1}, {"div", "Div", "DIV", 11, 0},
        {"curl", "Curl", "CURL", 12, 0}, {"Vr", "vr", "VR", 13, 0},
        {"Vtheta", "vtheta", "VTHETA", 14, 0}, {"trr", "TRR", "TRR", 15, 0},
        {"trtheta", "TRTHETA", "TRTHETA", 16, 0}, {"trz", "TRZ", "TRZ", 17, 0},
        {"tthetatheta", "TTHETATHETA", "TTHETATHETA", 18, 0},
        {"tthetaz", "TTHETAZ", "TTHETAZ", 19, 0},
    };
    for (size_t q = 0; q < sizeof tab / sizeof tab[0]; ++q)
        if ((!three_d || tab[q].in3d) &&
            (!strcmp(t, tab[q].a) || !strcmp(t, tab[q].b) || !strcmp(t, tab[q].c)))
            return tab[q].v;
    return -1;
}

int sm_read_records(const char *path, const sm_grid *g, int three_d, sm_record **out, size_t *nout)
{
    /* io_utils.c:1592-1682 (2-D) and 1684-1741 (3-D) */
    FILE *fid = fopen(path, "r");
    if (!fid) return sm_fail(SM_EIO, "cannot open %s for reading", path);
    size_t nrec = 0;
    if (fscanf(fid, "%zu", &nrec) != 1) {
        fclose(fid);
        return sm_fail(SM_EIO, "%s: bad record count", path);
    }
    sm_record *r = calloc(nrec ? nrec : 1, sizeof *r);
    if (!r) { fclose(fid); return sm_fail(SM_ENOMEM, "out of host memory"); }
    char t[80];
    for (size_t n = 0; n < nrec; ++n) {
        if (fscanf(fid, "%79s", t) != 1) goto bad;
        int c = record_comp(t, three_d);
        if (c < 0) {
            fclose(fid); free(r);
            return sm_fail(SM_EIO, "particle velocity component (%s) does not exists", t);
        }
        r[n].comp = c;
        if (fscanf(fid, "%79s", t) != 1) goto bad;
        if (!strcmp(t, "Trace") || !strcmp(t, "trace") || !strcmp(t, "TRACE")) {
            r[n].is_trace = 1;
            if (three_d) {
                if (fscanf(fid, "%lf %lf %lf", &r[n].x, &r[n].y, &r[n].z) != 3) goto bad;
            } else if (fscanf(fid, "%lf %lf", &r[n].x, &r[n].z) != 2) goto bad;
            if (fscanf(fid, "%lf", &r[n].t0) != 1 || fscanf(fid, "%lf", &r[n].dt) != 1) goto bad;
            r[n].dt *= 1.e-3;   /* ms -> s */
            r[n].i = c_round((r[n].x - g->x0) / g->dx);
            r[n].j = three_d ? c_round((r[n].y - g->y0) / g->dy) : 0;
            r[n].k = c_round((r[n].z - g->z0) / g->dz);
        } else if (!strcmp(t, "Snapshot") || !strcmp(t, "snapshot") || !strcmp(t, "SNAPSHOT")) {
            r[n].is_trace = 0;
            if (fscanf(fid, "%lf", &r[n].t0) != 1 || fscanf(fid, "%lf", &r[n].dt) != 1) goto bad;
            r[n].dt *= 1.e-3;
        } else {
            fclose(fid); free(r);
            return sm_fail(SM_EIO, "type of record (%s) not implemented", t);
        }
    }
    fclose(fid);
    *out = r;
    *nout = nrec;
    return SM_OK;
bad:
    fclose(fid);
    free(r);
    return sm_fail(SM_EIO, "something wrong with file %s", path);
}

static int ensure_dir(const char *d)
{
    struct stat sb;
    if (stat(d, &sb) == 0) return S_ISDIR(sb.st_mode) ? SM_OK : sm_fail(SM_EIO, "%s is not a directory", d);
    if (mkdir(d, S_IRWXU) != 0 && errno != EEXIST)
        return sm_fail(SM_EIO, "cannot create %s (%s)", d, strerror(errno));
    return SM_OK;
}

int sm_write_trace_file(const char *base, size_t n, const double *t, const double *v, size_t ns)
{
    /* io_utils.c:1744-1768 */
    char path[512];
    int rc;
    if ((rc = ensure_dir("trc"))) return rc;
    snprintf(path, sizeof path, "trc/%s", base);
    if ((rc = ensure_dir(path))) return rc;
    snprintf(path, sizeof path, "trc/%s/%s_%zu.trc", base, base, n);
    FILE *f = fopen(path, "w+");
    if (!f) return sm_fail(SM_EIO, "cannot open %s for output (%s)", path, strerror(errno));
    for (size_t s = 0; s < ns; ++s) fprintf(f, "%le    %le\n", t[s], 1.e3 * v[s]);
    if (fclose(f) != 0) return sm_fail(SM_EIO, "write error on %s", path);
    return SM_OK;
}

/* ---- the trace files of a run, written on host threads ---- */
typedef struct {
    const char *base;
    const size_t *recno, *counts;
    const double *t0, *rdt, *vals;
    double dt;
    size_t nsteps, ld, r0, r1;
    int rc;
    char msg[512];   /* the failing thread's message (messages are per thread) */
} trace_part;

static void *trace_files(void *arg)
{
    trace_part *w = (trace_part *)arg;
    w->rc = SM_OK;
    double *t = malloc((w->ld ? w->ld : 1) * sizeof(double));
    if (!t) {
        w->rc = SM_ENOMEM;
        snprintf(w->msg, sizeof w->msg, "out of host memory");
        return NULL;
    }
    for (size_t r = w->r0; r < w->r1; ++r) {
        /* the sample times: the steps the sampling test keeps (e_iso.c:641-669) */
        size_t s = 0;
        for (size_t it = 0; it < w->nsteps && s < w->counts[r]; ++it)
            if (sm_sample_predicate(it, w->dt, w->t0[r], w->rdt[r])) t[s++] = w->dt * (double)(it + 1);
        const int rc = sm_write_trace_file(w->base, w->recno[r] + 1, t, w->vals + r * w->ld,
                                           w->counts[r]);
        if (rc) {
            w->rc = rc;
            snprintf(w->msg, sizeof w->msg, "%s", sm_last_error());
            break;
        }
    }
    free(t);
    return NULL;
}

int sm_write_trace_set(const char *base, size_t nrec, const size_t *recno, const double *t0,
                       const double *rdt, double dt, size_t nsteps, const double *vals, size_t ld,
                       const size_t *counts)
{
    if (!nrec) return SM_OK;
    if (!base || !recno || !t0 || !rdt || !vals || !counts)
        return sm_fail(SM_EINVAL, "sm_write_trace_set: NULL argument");
    /* the directories first, so the threads only find them */
    char path[512];
    int rc;
    if ((rc = ensure_dir("trc"))) return rc;
    snprintf(path, sizeof path, "trc/%s", base);
    if ((rc = ensure_dir(path))) return rc;
    const size_t nt = sm_host_threads(nrec, 64);
    trace_part w[SM_MAX_HOST_THREADS];
    for (size_t k = 0; k < nt; ++k)
        w[k] = (trace_part){base, recno, counts, t0, rdt, vals, dt, nsteps, ld,
                            nrec * k / nt, nrec * (k + 1) / nt, SM_OK, {0}};
    sm_parallel(trace_files, w, sizeof w[0], nt);
    for (size_t k = 0; k < nt; ++k)   /* the first failure in receiver order */
        if (w[k].rc) return sm_fail(w[k].rc, "%s", w[k].msg);
    return SM_OK;
}

/* ---- SEG-Y (io_utils.c:3269-3559 layout) ---- */

static int put(FILE *f, const void *p, size_t n) { return fwrite(p, 1, n, f) == n; }
static int put16(FILE *f, int16_t v) { return put(f, &v, 2); }
static int put32(FILE *f, int32_t v) { return put(f, &v, 4); }
static int pad_to(FILE *f, long pos) {
    long cur = ftell(f);
    while (cur < pos) {
        if (fputc(0, f) == EOF) return 0;
        ++cur;
    }
    return 1;
}

static size_t segy_samples(const sm_params *p, double rdt)
{
    return (size_t)llround(p->duration / rdt) + 1;
}

int sm_write_segy(const char *base, const sm_params *p, const sm_record *rec, size_t ntr,
                  const sm_source *src0, const double *v, const double *t, size_t ld,
                  const size_t *count)
{
    char fname[600];
    struct stat sb;
    if (stat("segy", &sb) < 0 && errno == ENOENT) mkdir("segy", S_IRWXU);
    snprintf(fname, sizeof fname, "segy/%s.sgy", base);
    FILE *f = fopen(fname, "wb");
    if (!f) return sm_fail(SM_EIO, "cannot open %s for output (%s)", fname, strerror(errno));
    int ok = 1;
    /* textual file header: blanks with 'C' in columns 1 of the first two cards */
    char text[3200];
    memset(text, ' ', sizeof text);
    text[0] = 'C';
    text[80] = 'C';
    ok = ok && put(f, text, sizeof text);
    /* binary file header (fields 1-26, then the revision block at 3500) */
    int16_t dt_us = 0, ns0 = 0, fold = 0;
    if (ntr) {
        dt_us = (int16_t)(1000000 * rec[0].dt);
        ns0 = (int16_t)segy_samples(p, rec[0].dt);
    }
    for (size_t r = 0; r < ntr; ++r) fold += rec[r].comp == SM_VZ;
    if (fold == 0)
        for (size_t r = 0; r < ntr; ++r) fold += rec[r].comp == SM_VY;
    ok = ok && put32(f, 1) && put32(f, 1) && put32(f, 1);     /* job, line, reel */
    ok = ok && put16(f, (int16_t)ntr) && put16(f, 0);          /* traces, aux traces */
    ok = ok && put16(f, dt_us) && put16(f, dt_us);             /* sample interval (us) */
    ok = ok && put16(f, ns0) && put16(f, ns0);                 /* samples per trace */
    ok = ok && put16(f, 5);                                    /* IEEE float32 */
    ok = ok && put16(f, fold) && put16(f, 1) && put16(f, 1);   /* fold, sorting, vertical sum */
    for (int k = 14; k <= 23; ++k) ok = ok && put16(f, 0);
    ok = ok && put16(f, 1) && put16(f, 1) && put16(f, 1);      /* amp. recovery, units, polarity */
    ok = ok && pad_to(f, 3500);
    ok = ok && put16(f, 1) && put16(f, 0) && put16(f, 0);      /* rev. 1, fixed-length flag, ext. hdrs */
    ok = ok && pad_to(f, 3600);
    time_t now = time(NULL);
    struct tm *tm_now = gmtime(&now);
    int32_t src_no = p->shotpt_no;
    const double sx = src0 ? src0->x : 0.0, sz = src0 ? src0->z : 0.0;
    for (size_t r = 0; r < ntr && ok; ++r) {
        const sm_record *q = &rec[r];
        const int32_t tr_no = (int32_t)(r + 1);
        const long start = ftell(f);
        ok = ok && put32(f, tr_no) && put32(f, tr_no) && put32(f, tr_no) && put32(f, tr_no);
        ok = ok && put32(f, src_no) && put32(f, 1) && put32(f, tr_no);
        if (p->simulate_cmp) src_no++;
        int16_t code = 1;
        if (q->comp == SM_VZ) code = 12;
        else if (q->comp == SM_VY) code = 13;
        else if (q->comp == SM_VX) code = 14;
        else if (q->comp == SM_P) code = 11;
        ok = ok && put16(f, code) && put16(f, 1) && put16(f, 1) && put16(f, 1);
        const int32_t offset = (int32_t)(q->x - sx);
        ok = ok && put32(f, offset) && put32(f, (int32_t)(-q->z)) && put32(f, 0) &&
             put32(f, (int32_t)(sz - 0));
        for (int k = 0; k < 4; ++k) ok = ok && put32(f, 0);
        ok = ok && put16(f, 1) && put16(f, 1);
        ok = ok && put32(f, p->simulate_cmp ? -offset / 2 : (int32_t)sx) && put32(f, 0);
        ok = ok && put32(f, p->simulate_cmp ? offset / 2 : (int32_t)q->x) && put32(f, 0);
        ok = ok && put16(f, 1) && put16(f, 500) && put16(f, 500);
        for (int k = 0; k < 10; ++k) ok = ok && put16(f, 0);
        const size_t ns = segy_samples(p, q->dt);
        ok = ok && put16(f, (int16_t)ns) && put16(f, (int16_t)(1000000 * q->dt));
        ok = ok && put16(f, 1) && put16(f, 1) && put16(f, 1);
        for (int k = 0; k < 16; ++k) ok = ok && put16(f, 0);
        ok = ok && put16(f, (int16_t)(1900 + tm_now->tm_year)) && put16(f, (int16_t)tm_now->tm_yday) &&
             put16(f, (int16_t)tm_now->tm_hour) && put16(f, (int16_t)tm_now->tm_min) &&
             put16(f, (int16_t)tm_now->tm_sec) && put16(f, 2);
        for (int k = 0; k < 5; ++k) ok = ok && put16(f, 0);
        ok = ok && put16(f, 2);
        ok = ok && put32(f, offset);
        for (int k = 0; k < 4; ++k) ok = ok && put32(f, 0);
        ok = ok && put16(f, 1) && put16(f, 6) && put32(f, 1) && put16(f, 0) && put16(f, 6) &&
             put16(f, 0) && put16(f, 1) && put16(f, 4);
        ok = ok && pad_to(f, start + 240);
        float *data = calloc(ns, sizeof(float));
        if (!data) {
            fclose(f);
            return sm_fail(SM_ENOMEM, "out of host memory");
        }
        for (size_t k = 0; k < count[r]; ++k) {
            const size_t i = (size_t)llround(t[r * ld + k] / q->dt);
            if (i < ns) data[i] = (float)v[r * ld + k];
        }
        ok = ok && put(f, data, ns * sizeof(float));
        free(data);
    }
    if (fclose(f) != 0) ok = 0;
    if (!ok) return sm_fail(SM_EIO, "write error on %s", fname);
    return SM_OK;
}

/* the snapshot file of write_snapshot; npl: absorbing columns before column
 * 0 of the model (np on the Cartesian grids, 0 on the cylindrical one, whose
 * axis has none), npr: after its last column */
/* one thread's share of a text snapshot: the lines of columns [i0, i1),
 * formatted into its own buffer (the bytes fprintf would write) */
typedef struct {
    const double *data;
    size_t nx2, nz2, npl, npr, np, i0, i1;
    double dx, dz, x0, z0;
    int plot_strips;
    char *buf;
    size_t len, cap;
    int bad;
} snap_part;

static void snap_put(snap_part *w, double x, double z, double v)
{
    if (w->bad) return;
    if (w->cap - w->len < 128) {
        size_t cap = w->cap ? 2 * w->cap : (size_t)1 << 16;
        char *nb = realloc(w->buf, cap);
        if (!nb) { w->bad = 1; return; }
        w->buf = nb;
        w->cap = cap;
    }
    const int k = snprintf(w->buf + w->len, w->cap - w->len, "%le  %le  %le\n", x, z, v);
    if (k < 0 || (size_t)k >= w->cap - w->len) { w->bad = 1; return; }
    w->len += (size_t)k;
}

static void *snap_format(void *arg)
{
    snap_part *w = (snap_part *)arg;
    for (size_t i = w->i0; i < w->i1; ++i) {
        if (w->plot_strips) {
            const double x = w->x0 + ((double)i - (double)w->npl) * w->dx;
            for (size_t k = 0; k < w->nz2; ++k)
                snap_put(w, x, w->z0 + ((double)k - (double)w->np) * w->dz,
                         1.e3 * w->data[i * w->nz2 + k]);
        } else {
            const double x = w->x0 + i * w->dx;
            for (size_t k = 0; k + 2 * w->np < w->nz2; ++k)
                snap_put(w, x, w->z0 + k * w->dz, 1.e3 * w->data[(i + w->npl) * w->nz2 + k + w->np]);
        }
    }
    return NULL;
}

/* write_snapshot (io_utils.c:1775-1820): "x  z  1e3*v" per node, the
 * interior or with plot_strips the whole padded grid; the columns are
 * formatted on host threads and written in order */
static int write_snapshot_grid(const char *base, size_t n, double t, const double *data,
                               size_t nx2, size_t nz2, size_t npl, size_t npr, size_t np,
                               double dx, double dz, double x0, double z0, int plot_strips)
{
    char name[700];
    struct stat sb;
    if (stat("ssh", &sb) < 0 && errno == ENOENT) mkdir("ssh", S_IRWXU);
    snprintf(name, sizeof name, "ssh/%s", base);
    if (stat(name, &sb) < 0 && errno == ENOENT) mkdir(name, S_IRWXU);
    snprintf(name, sizeof name, "ssh/%s/%s_%zu_%lf.ssh", base, base, n, t);
    FILE *f = fopen(name, "w");
    if (!f) return sm_fail(SM_EIO, "cannot open %s for output (%s)", name, strerror(errno));
    const size_t ncol = plot_strips ? nx2 : (nx2 > npl + npr ? nx2 - npl - npr : 0);
    size_t nt = sm_host_threads(ncol * nz2, (size_t)1 << 16);
    if (nt > ncol) nt = ncol ? ncol : 1;
    snap_part w[SM_MAX_HOST_THREADS];
    for (size_t k = 0; k < nt; ++k)
        w[k] = (snap_part){data, nx2, nz2, npl, npr, np, ncol * k / nt, ncol * (k + 1) / nt,
                           dx, dz, x0, z0, plot_strips, NULL, 0, 0, 0};
    sm_parallel(snap_format, w, sizeof w[0], nt);
    int ok = 1;
    for (size_t k = 0; k < nt; ++k) {
        if (w[k].bad) ok = 0;
        if (ok && w[k].len && fwrite(w[k].buf, 1, w[k].len, f) != w[k].len) ok = 0;
        free(w[k].buf);
    }
    if (fclose(f) != 0) ok = 0;
    return ok ? SM_OK : sm_fail(SM_EIO, "write error on %s", name);
}

int sm_write_snapshot(const char *base, size_t n, double t, const double *data, size_t nx2,
                      size_t nz2, size_t np, double dx, double dz, double x0, double z0,
                      int plot_strips)
{
    return write_snapshot_grid(base, n, t, data, nx2, nz2, np, np, np, dx, dz, x0, z0,
                               plot_strips);
}

int sm_write_snapshot_cyl(const char *base, size_t n, double t, const double *data, size_t nx2,
                          size_t nz2, size_t np, double dx, double dz, double x0, double z0,
                          int plot_strips)
{
    return write_snapshot_grid(base, n, t, data, nx2, nz2, 0, np, np, dx, dz, x0, z0,
                               plot_strips);
}
