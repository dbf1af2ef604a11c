/*
 * pscf_oracle.c -- FP64 CPU oracle for the PSCF propagator hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA engine
 * (pscf_b200/csrc) is compared against.  Only tests/, the smoke check in
 * __graft_entry__.py and the cpu_baseline leg of bench.py may load it.  The
 * product path never links, loads or calls anything built from here.
 *
 * It is a from-the-mathematics restatement (plain C99, no FFTW) of the
 * reference Fortran routines listed below; every function names the
 * reference file:line it follows.  The FFT is a self-written mixed-radix
 * transform standing in for FFTW (third-party, not vendored in the
 * reference; FFTW >= 3.3.0 per CMakeLists.txt:111-119).  It has FFTW's
 * sign and normalisation conventions: forward e^{-i}, unnormalised;
 * inverse e^{+i}, unnormalised (src/fft3_mod.f90:85-122).
 *
 * Grid storage follows the reference: x fastest (Fortran column-major), so a
 * real field is double[n3][n2][n1]; the r2c half spectrum is
 * complex[n3][n2][n1/2+1] (src/grid_mod.f90:103-110, src/step_mod.f90:73-80).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>
#include <stdio.h>
#include <pthread.h>

typedef double complex cplx;

#define ORC_MAXM 4      /* monomer types   */
#define ORC_MAXC 4      /* chain species   */
#define ORC_MAXB 8      /* blocks / chain  */
#define ORC_MAXS 4      /* solvent species */
#define ORC_MAXCP 6     /* cell parameters */

/* Physical system: mirrors the module globals the reference reads
 * (src/chemistry_mod.f90:41-46, src/grid_mod.f90:43-46,
 * src/unit_cell_mod.f90 R_basis/G_basis/dGG_basis). */
typedef struct {
    int dim;
    int n[3];
    int n_monomer;
    int n_chain;
    int n_solvent;
    int ensemble;                 /* 0 canonical, 1 grand */
    int n_block[ORC_MAXC];
    int block_monomer[ORC_MAXC][ORC_MAXB];   /* 0-based monomer index */
    double block_length[ORC_MAXC][ORC_MAXB];
    double kuhn[ORC_MAXM];
    double chi[ORC_MAXM][ORC_MAXM];
    double phi_chain[ORC_MAXC];
    double mu_chain[ORC_MAXC];
    int solvent_monomer[ORC_MAXS];
    double solvent_size[ORC_MAXS];
    double phi_solvent[ORC_MAXS];
    double mu_solvent[ORC_MAXS];
    double ds;                    /* chain_step */
    double G_basis[3][3];         /* row i = reciprocal basis vector i */
    int n_cell_param;
    double dGG[ORC_MAXCP][3][3];  /* d(b_i . b_j)/d(cell_param k) */
} orc_system;

/* ------------------------------------------------------------------ */
/* Mixed-radix complex FFT (recursive decimation in time).             */
/* ------------------------------------------------------------------ */

typedef struct {
    int n;
    int nf;
    int fac[40];
    cplx *tw;        /* tw[j] = exp(-2 pi i j / n) */
} fft1d;

static int fft1d_init(fft1d *p, int n)
{
    p->n = n;
    p->nf = 0;
    int m = n;
    const int pref[] = {4, 2, 3, 5, 7};
    while (m > 1) {
        int found = 0;
        for (int i = 0; i < 5; i++) {
            if (m % pref[i] == 0) { p->fac[p->nf++] = pref[i]; m /= pref[i]; found = 1; break; }
        }
        if (!found) {
            /* generic prime factor */
            int f = 11;
            while (m % f) f += 2;
            p->fac[p->nf++] = f;
            m /= f;
        }
    }
    p->tw = (cplx *)malloc(sizeof(cplx) * (n > 0 ? n : 1));
    for (int j = 0; j < n; j++) {
        /* angle reduced exactly in integers before the trig call */
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)j / (long double)n;
        p->tw[j] = (double)cosl(a) + I * (double)sinl(a);
    }
    return 0;
}

static void fft1d_free(fft1d *p) { free(p->tw); p->tw = NULL; }

/* out[0..n) = DFT of in[0], in[stride], ...; twiddles W_N^(j*tws) where N is
 * the top-level length.  sign=-1 forward, +1 inverse. */
static void fft_rec(const cplx *in, cplx *out, int n, int stride, const int *fac,
                    const cplx *tw, int tws, int N, int sign)
{
    if (n == 1) { out[0] = in[0]; return; }
    int p = fac[0];
    int m = n / p;
    for (int r = 0; r < p; r++)
        fft_rec(in + (long)r * stride, out + (long)r * m, m, stride * p, fac + 1, tw, tws * p, N, sign);
    cplx t[64];
    cplx y[64];
    for (int k = 0; k < m; k++) {
        for (int r = 0; r < p; r++) {
            cplx w = tw[((long)r * k * tws) % N];
            if (sign > 0) w = conj(w);
            t[r] = out[(long)r * m + k] * w;
        }
        for (int q = 0; q < p; q++) {
            cplx s = 0;
            for (int r = 0; r < p; r++) {
                cplx w = tw[((long)((r * q) % p) * m * tws) % N];
                if (sign > 0) w = conj(w);
                s += t[r] * w;
            }
            y[q] = s;
        }
        for (int q = 0; q < p; q++) out[k + (long)q * m] = y[q];
    }
}

static void fft1d_exec(const fft1d *p, const cplx *in, cplx *out, int sign)
{
    fft_rec(in, out, p->n, 1, p->fac, p->tw, 1, p->n, sign);
}

/* 3-D plan: full complex transforms used to build r2c / c2r. */
typedef struct {
    int n[3];
    long nr;            /* n1*n2*n3 */
    long nk;            /* (n1/2+1)*n2*n3 */
    int n1h;
    fft1d p[3];
    cplx *full;         /* nr complex */
    cplx *lin, *lout;   /* line buffers */
} fft3d;

static void fft3d_init(fft3d *f, const int n[3])
{
    int mx = 1;
    for (int i = 0; i < 3; i++) {
        f->n[i] = n[i];
        fft1d_init(&f->p[i], n[i]);
        if (n[i] > mx) mx = n[i];
    }
    f->nr = (long)n[0] * n[1] * n[2];
    f->n1h = n[0] / 2 + 1;
    f->nk = (long)f->n1h * n[1] * n[2];
    f->full = (cplx *)malloc(sizeof(cplx) * f->nr);
    f->lin = (cplx *)malloc(sizeof(cplx) * mx);
    f->lout = (cplx *)malloc(sizeof(cplx) * mx);
}

static void fft3d_free(fft3d *f)
{
    for (int i = 0; i < 3; i++) fft1d_free(&f->p[i]);
    free(f->full); free(f->lin); free(f->lout);
}

/* Threads of the 3-D transforms (POSIX threads over independent lines; 1 =
 * serial).  The lines are independent, so the result does not depend on it. */
static int g_fft_threads = 1;

int orc_set_fft_threads(int n)
{
    g_fft_threads = n < 1 ? 1 : (n > 64 ? 64 : n);
    return 0;
}

typedef struct {
    fft3d *f;
    cplx *a;
    int sign, axis;
    long l0, l1;   /* line range */
} lines_job;

/* Lines [l0, l1) along one axis: x lines are numbered l = j + n2 k, y lines
 * l = i + n1 k, z lines l = i + n1 j. */
static void *lines_run(void *arg)
{
    lines_job *J = (lines_job *)arg;
    fft3d *f = J->f;
    const int n1 = f->n[0], n2 = f->n[1];
    const int ax = J->axis, n = f->n[ax];
    cplx *lin = (cplx *)malloc(sizeof(cplx) * n), *lout = (cplx *)malloc(sizeof(cplx) * n);
    for (long l = J->l0; l < J->l1; l++) {
        long base, es;
        if (ax == 0) { base = l * n1; es = 1; }
        else if (ax == 1) { base = (l % n1) + (long)n1 * n2 * (l / n1); es = n1; }
        else { base = l; es = (long)n1 * n2; }
        for (int e = 0; e < n; e++) lin[e] = J->a[base + e * es];
        fft1d_exec(&f->p[ax], lin, lout, J->sign);
        for (int e = 0; e < n; e++) J->a[base + e * es] = lout[e];
    }
    free(lin);
    free(lout);
    return NULL;
}

static void fft3d_lines(fft3d *f, cplx *a, int sign, int axis)
{
    const long nl = f->nr / f->n[axis];
    int nt = g_fft_threads;
    if (nt > nl) nt = (int)nl;
    lines_job jobs[64];
    pthread_t th[64];
    for (int t = 0; t < nt; t++) {
        jobs[t].f = f;
        jobs[t].a = a;
        jobs[t].sign = sign;
        jobs[t].axis = axis;
        jobs[t].l0 = nl * t / nt;
        jobs[t].l1 = nl * (t + 1) / nt;
    }
    if (nt <= 1) {
        lines_run(&jobs[0]);
        return;
    }
    for (int t = 1; t < nt; t++) pthread_create(&th[t], NULL, lines_run, &jobs[t]);
    lines_run(&jobs[0]);
    for (int t = 1; t < nt; t++) pthread_join(th[t], NULL);
}

static void fft3d_c2c_inplace(fft3d *f, cplx *a, int sign)
{
    for (int ax = 0; ax < 3; ax++)
        if (f->n[ax] > 1) fft3d_lines(f, a, sign, ax);
}

/* r2c forward, unnormalised (FFTW dfftw_plan_dft_r2c_3d, src/fft3_mod.f90:85-94) */
static void fft3d_r2c(fft3d *f, const double *in, cplx *out)
{
    for (long i = 0; i < f->nr; i++) f->full[i] = in[i];
    fft3d_c2c_inplace(f, f->full, -1);
    const int n1 = f->n[0], n1h = f->n1h;
    for (long l = 0; l < (long)f->n[1] * f->n[2]; l++)
        for (int i = 0; i < n1h; i++) out[l * n1h + i] = f->full[l * n1 + i];
}

/* c2r inverse, unnormalised (FFTW dfftw_plan_dft_c2r_3d, src/fft3_mod.f90:113-122).
 * The missing half is rebuilt from Hermitian symmetry X(-k) = conj X(k). */
static void fft3d_c2r(fft3d *f, const cplx *in, double *out)
{
    const int n1 = f->n[0], n2 = f->n[1], n3 = f->n[2], n1h = f->n1h;
    for (int k = 0; k < n3; k++)
        for (int j = 0; j < n2; j++)
            for (int i = 0; i < n1; i++) {
                cplx v;
                if (i < n1h) v = in[i + (long)n1h * (j + (long)n2 * k)];
                else {
                    int ii = n1 - i, jj = (n2 - j) % n2, kk = (n3 - k) % n3;
                    v = conj(in[ii + (long)n1h * (jj + (long)n2 * kk)]);
                }
                f->full[i + (long)n1 * (j + (long)n2 * k)] = v;
            }
    fft3d_c2c_inplace(f, f->full, +1);
    for (long i = 0; i < f->nr; i++) out[i] = creal(f->full[i]);
}

/* Exported thin wrappers so tests can pin the FFT against numpy.fft. */
int orc_fft_r2c(const int n[3], const double *in, double *out_interleaved)
{
    fft3d f;
    fft3d_init(&f, n);
    fft3d_r2c(&f, in, (cplx *)out_interleaved);
    fft3d_free(&f);
    return 0;
}

int orc_fft_c2r(const int n[3], const double *in_interleaved, double *out)
{
    fft3d f;
    fft3d_init(&f, n);
    fft3d_c2r(&f, (const cplx *)in_interleaved, out);
    fft3d_free(&f);
    return 0;
}

int orc_fft_c2c(const int n[3], double *inout_interleaved, int sign)
{
    fft3d f;
    fft3d_init(&f, n);
    fft3d_c2c_inplace(&f, (cplx *)inout_interleaved, sign);
    fft3d_free(&f);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Grid geometry: k^2 table (src/grid_mod.f90:141-160, 225-283, 394-405) */
/* ------------------------------------------------------------------ */

/* |G|^2 for integer wave G with Gvec = sum_i G(i) G_basis(i,:)
 * (src/grid_mod.f90:394-405 norm, ivec .dot. mat contracts the first index) */
static double g_norm(int dim, const int G[3], const double Gb[3][3])
{
    double v[3] = {0, 0, 0};
    for (int j = 0; j < dim; j++)
        for (int i = 0; i < dim; i++) v[j] += G[i] * Gb[i][j];
    double s = 0;
    for (int j = 0; j < dim; j++) s += v[j] * v[j];
    return s;
}

/* Minimum-image wave: shifts tried in the order +1, 0, -1 for each used
 * dimension, a later image replaces the kept one only when smaller by more
 * than 1e-8 (src/grid_mod.f90:225-283). */
void orc_G_to_bz(int dim, const int n[3], const double Gb[3][3], const int G[3], int out[3])
{
    int Gmin[3] = {0, 0, 0}, Gt[3] = {0, 0, 0};
    double gmin = 1.0e10;
    const double delta = 1.0e-8;
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) { lo[d] = -1; hi[d] = 1; }
    for (int i1 = hi[0]; i1 >= lo[0]; i1--) {
        Gt[0] = G[0] + i1 * n[0];
        for (int i2 = hi[1]; i2 >= lo[1]; i2--) {
            Gt[1] = (dim > 1) ? G[1] + i2 * n[1] : 0;
            for (int i3 = hi[2]; i3 >= lo[2]; i3--) {
                Gt[2] = (dim > 2) ? G[2] + i3 * n[2] : 0;
                double g = g_norm(dim, Gt, Gb);
                if (g < gmin - delta) {
                    for (int d = 0; d < dim; d++) Gmin[d] = Gt[d];
                    gmin = g;
                }
            }
        }
    }
    out[0] = Gmin[0]; out[1] = Gmin[1]; out[2] = Gmin[2];
}

/* ksq(0:n1/2, 0:n2-1, 0:n3-1) (src/grid_mod.f90:141-160).  Optionally also
 * the folded integer waves (3 ints per k point) used by the stress. */
void orc_make_ksq(int dim, const int n[3], const double Gb[3][3], double *ksq, int *gbz)
{
    const int n1h = n[0] / 2 + 1;
    for (int i3 = 0; i3 < n[2]; i3++)
        for (int i2 = 0; i2 < n[1]; i2++)
            for (int i1 = 0; i1 < n1h; i1++) {
                int G[3] = {i1, i2, i3}, Gz[3];
                orc_G_to_bz(dim, n, Gb, G, Gz);
                long idx = i1 + (long)n1h * (i2 + (long)n[1] * i3);
                ksq[idx] = g_norm(dim, Gz, Gb);
                if (gbz) { gbz[3 * idx] = Gz[0]; gbz[3 * idx + 1] = Gz[1]; gbz[3 * idx + 2] = Gz[2]; }
            }
}

/* ------------------------------------------------------------------ */
/* Contour discretisation (src/chain_mod.f90:136-158)                   */
/* ------------------------------------------------------------------ */

/* block_bgn is 1-based like the reference: block i spans slices
 * block_bgn[i] .. block_bgn[i+1] (inclusive); returns total slices. */
int orc_chain_grid(int nblk, const double *blk_length, double ds, int *block_bgn, double *block_ds)
{
    int bgns = 1;
    block_bgn[0] = bgns;
    for (int i = 0; i < nblk; i++) {
        int iblk = (int)(blk_length[i] / ds / 2.0 + 0.5);
        if (iblk == 0) {
            iblk = 1;
            block_ds[i] = blk_length[i] / 2.0;
        } else {
            block_ds[i] = blk_length[i] / (double)iblk / 2.0;
        }
        bgns += iblk * 2;
        block_bgn[i + 1] = bgns;
    }
    return bgns;
}

/* ------------------------------------------------------------------ */
/* Propagator (src/step_mod.f90:109-176)                                */
/* ------------------------------------------------------------------ */

typedef struct {
    fft3d f;
    long nr, nk;
    double *eo1, *eo2, *ek1, *ek2;
    double *qr, *q1, *q2;
    cplx *qk;
} stepper;

static void stepper_init(stepper *s, const int n[3])
{
    fft3d_init(&s->f, n);
    s->nr = s->f.nr; s->nk = s->f.nk;
    s->eo1 = malloc(sizeof(double) * s->nr);
    s->eo2 = malloc(sizeof(double) * s->nr);
    s->ek1 = malloc(sizeof(double) * s->nk);
    s->ek2 = malloc(sizeof(double) * s->nk);
    s->qr = malloc(sizeof(double) * s->nr);
    s->q1 = malloc(sizeof(double) * s->nr);
    s->q2 = malloc(sizeof(double) * s->nr);
    s->qk = malloc(sizeof(cplx) * s->nk);
}

static void stepper_free(stepper *s)
{
    fft3d_free(&s->f);
    free(s->eo1); free(s->eo2); free(s->ek1); free(s->ek2);
    free(s->qr); free(s->q1); free(s->q2); free(s->qk);
}

/* make_propg (src/step_mod.f90:109-129) */
static void make_propg(stepper *s, double ds, double b, const double *ksq, const double *omega)
{
    double lap = ds * (b * b) / 6.0;
    double pot = ds / 2.0;
    for (long k = 0; k < s->nk; k++) {
        s->ek1[k] = exp(-lap * ksq[k]);
        s->ek2[k] = exp(-(lap / 2.0) * ksq[k]);
    }
    for (long r = 0; r < s->nr; r++) {
        s->eo1[r] = exp(-pot * omega[r]);
        s->eo2[r] = exp(-(pot / 2.0) * omega[r]);
    }
}

/* step_exp (src/step_mod.f90:146-176): one full step q1, two half steps q2,
 * Richardson combination (4 q2 - q1)/3. */
static void step_exp(stepper *s, const double *qin, double *qout)
{
    const long nr = s->nr, nk = s->nk;
    const double rn = (double)nr;
    for (long r = 0; r < nr; r++) s->qr[r] = s->eo1[r] * qin[r];
    fft3d_r2c(&s->f, s->qr, s->qk);
    for (long k = 0; k < nk; k++) s->qk[k] *= s->ek1[k];
    fft3d_c2r(&s->f, s->qk, s->qr);
    for (long r = 0; r < nr; r++) s->q1[r] = s->eo1[r] * s->qr[r] / rn;

    for (long r = 0; r < nr; r++) s->qr[r] = s->eo2[r] * qin[r];
    fft3d_r2c(&s->f, s->qr, s->qk);
    for (long k = 0; k < nk; k++) s->qk[k] *= s->ek2[k];
    fft3d_c2r(&s->f, s->qk, s->qr);
    for (long r = 0; r < nr; r++) s->qr[r] = s->eo1[r] * s->qr[r] / rn;
    fft3d_r2c(&s->f, s->qr, s->qk);
    for (long k = 0; k < nk; k++) s->qk[k] *= s->ek2[k];
    fft3d_c2r(&s->f, s->qk, s->qr);
    for (long r = 0; r < nr; r++) s->q2[r] = s->eo2[r] * s->qr[r] / rn;

    for (long r = 0; r < nr; r++) qout[r] = (4.0 * s->q2[r] - s->q1[r]) / 3.0;
}

/* Exported single step for parity tests. */
int orc_step(const int n[3], const double *ksq, double b, double ds,
             const double *omega, const double *qin, double *qout, int nsteps)
{
    stepper s;
    stepper_init(&s, n);
    make_propg(&s, ds, b, ksq, omega);
    double *tmp = malloc(sizeof(double) * s.nr);
    memcpy(tmp, qin, sizeof(double) * s.nr);
    for (int i = 0; i < nsteps; i++) {
        step_exp(&s, tmp, qout);
        memcpy(tmp, qout, sizeof(double) * s.nr);
    }
    free(tmp);
    stepper_free(&s);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Chain density (src/scf_mod.fp.f90:315-426)                           */
/* ------------------------------------------------------------------ */

typedef struct {
    int nblk;
    int ns;                     /* total slices = block_bgn[nblk] */
    int block_bgn[ORC_MAXB + 1];
    double block_ds[ORC_MAXB];
    double length;
    double *qf, *qr;            /* ns slices each */
    double *rho;                /* nblk fields */
    double bigQ;
} chain_work;

static void chain_work_init(chain_work *c, const orc_system *sys, int ic, long nr)
{
    c->nblk = sys->n_block[ic];
    c->ns = orc_chain_grid(c->nblk, sys->block_length[ic], sys->ds, c->block_bgn, c->block_ds);
    c->length = 0;
    for (int b = 0; b < c->nblk; b++) c->length += sys->block_length[ic][b];
    c->qf = malloc(sizeof(double) * nr * c->ns);
    c->qr = malloc(sizeof(double) * nr * c->ns);
    c->rho = malloc(sizeof(double) * nr * c->nblk);
}

static void chain_work_free(chain_work *c) { free(c->qf); free(c->qr); free(c->rho); }

static void chain_density(stepper *s, const orc_system *sys, int ic, chain_work *c,
                          const double *ksq, const double *omega)
{
    const long nr = s->nr;
    /* slice index (1-based in reference) j -> offset (j-1)*nr */
#define QF(j) (c->qf + (long)((j) - 1) * nr)
#define QR(j) (c->qr + (long)((j) - 1) * nr)
    for (long r = 0; r < nr; r++) QF(1)[r] = 1.0;
    for (int ib = 0; ib < c->nblk; ib++) {
        int mon = sys->block_monomer[ic][ib];
        make_propg(s, c->block_ds[ib], sys->kuhn[mon], ksq, omega + (long)mon * nr);
        for (int is = c->block_bgn[ib]; is <= c->block_bgn[ib + 1] - 1; is++)
            step_exp(s, QF(is), QF(is + 1));
    }
    int chain_end = c->block_bgn[c->nblk];
    for (long r = 0; r < nr; r++) QR(chain_end)[r] = 1.0;
    for (int ib = c->nblk - 1; ib >= 0; ib--) {
        int mon = sys->block_monomer[ic][ib];
        make_propg(s, c->block_ds[ib], sys->kuhn[mon], ksq, omega + (long)mon * nr);
        for (int is = c->block_bgn[ib + 1]; is >= c->block_bgn[ib] + 1; is--)
            step_exp(s, QR(is), QR(is - 1));
    }
    double sum = 0;
    for (long r = 0; r < nr; r++) sum += QF(chain_end)[r];
    c->bigQ = sum / (double)nr;

    for (int ib = 0; ib < c->nblk; ib++) {
        double *rho = c->rho + (long)ib * nr;
        int ibgn = c->block_bgn[ib], iend = c->block_bgn[ib + 1];
        for (long r = 0; r < nr; r++) rho[r] = QF(ibgn)[r] * QR(ibgn)[r];
        for (long r = 0; r < nr; r++) rho[r] = rho[r] + QF(iend)[r] * QR(iend)[r];
        for (int j = ibgn + 1; j <= iend - 1; j += 2)
            for (long r = 0; r < nr; r++) rho[r] = rho[r] + QF(j)[r] * QR(j)[r] * 4.0;
        for (int j = ibgn + 2; j <= iend - 2; j += 2)
            for (long r = 0; r < nr; r++) rho[r] = rho[r] + QF(j)[r] * QR(j)[r] * 2.0;
        for (long r = 0; r < nr; r++) rho[r] = rho[r] * c->block_ds[ib] / 3.0;
    }
    for (long r = 0; r < nr * c->nblk; r++) c->rho[r] = c->rho[r] / c->length / c->bigQ;
#undef QF
#undef QR
}

/* ------------------------------------------------------------------ */
/* Solver context                                                       */
/* ------------------------------------------------------------------ */

typedef struct {
    orc_system sys;
    long nr, nk;
    stepper st;
    chain_work ch[ORC_MAXC];
    double *ksq;
    int *gbz;
    double qout[ORC_MAXC];
    double qsolv[ORC_MAXS];
    double *kweight;    /* [nk] star-basis weights r(G) (1 without a group) */
    int nops;           /* space-group elements (0: no symmetry imposed) */
    int *symM;          /* [nops][3][3] integer action on grid indices   */
    int *symt;          /* [nops][3] translation in grid units           */
} orc_ctx;

orc_ctx *orc_create(const orc_system *sys)
{
    orc_ctx *c = calloc(1, sizeof(orc_ctx));
    c->sys = *sys;
    for (int d = sys->dim; d < 3; d++) c->sys.n[d] = 1;
    stepper_init(&c->st, c->sys.n);
    c->nr = c->st.nr; c->nk = c->st.nk;
    for (int i = 0; i < sys->n_chain; i++) chain_work_init(&c->ch[i], &c->sys, i, c->nr);
    c->ksq = malloc(sizeof(double) * c->nk);
    c->gbz = malloc(sizeof(int) * 3 * c->nk);
    orc_make_ksq(c->sys.dim, c->sys.n, c->sys.G_basis, c->ksq, c->gbz);
    return c;
}

void orc_destroy(orc_ctx *c)
{
    if (!c) return;
    stepper_free(&c->st);
    for (int i = 0; i < c->sys.n_chain; i++) chain_work_free(&c->ch[i]);
    free(c->ksq); free(c->gbz);
    free(c->symM); free(c->symt); free(c->kweight);
    free(c);
}

/* Space-group projection on the grid.  The reference keeps fields in a
 * symmetry-adapted star basis (src/basis_mod.f90, src/grid_basis_mod.f90);
 * on the grid the same subspace is reached by averaging f over the orbit
 * i -> M i + t (mod n) of every grid point. */
void orc_set_symmetry(orc_ctx *c, int nops, const int *M, const int *t)
{
    free(c->symM); free(c->symt);
    c->symM = NULL; c->symt = NULL;
    c->nops = nops;
    if (nops <= 0) { c->nops = 0; free(c->kweight); c->kweight = NULL; return; }
    c->symM = malloc(sizeof(int) * 9 * nops);
    c->symt = malloc(sizeof(int) * 3 * nops);
    memcpy(c->symM, M, sizeof(int) * 9 * nops);
    memcpy(c->symt, t, sizeof(int) * 3 * nops);
    /* Star weights.  A star is the orbit of a wave G under the point group,
     * G -> G.m (src/group_mod.f90:77-78), on the FFT grid.  The reference
     * normalises the star coefficients by sqrt(real(star_N)), a
     * single-precision square root (src/basis_mod.f90:920), so every star
     * sum over basis coefficients (free energy, stress) weights the star by
     * r = fl32(sqrt(N))^2 / N instead of 1. */
    const int *n = c->sys.n;
    const int n1h = n[0] / 2 + 1;
    if (!c->kweight) c->kweight = malloc(sizeof(double) * c->nk);
    long *seen = malloc(sizeof(long) * nops);
    for (int i3 = 0; i3 < n[2]; i3++)
        for (int i2 = 0; i2 < n[1]; i2++)
            for (int i1 = 0; i1 < n1h; i1++) {
                int G[3] = {i1, i2, i3};
                int cnt = 0;
                for (int k = 0; k < nops; k++) {
                    const int *m = M + 9 * k;
                    long key = 0;
                    for (int j = 0; j < 3; j++) {
                        long v = 0;
                        for (int i = 0; i < 3; i++) v += (long)G[i] * m[3 * i + j];
                        v %= n[j];
                        if (v < 0) v += n[j];
                        key = key * n[j] + v;
                    }
                    int dup = 0;
                    for (int q = 0; q < cnt; q++) if (seen[q] == key) { dup = 1; break; }
                    if (!dup) seen[cnt++] = key;
                }
                float sf = sqrtf((float)cnt);
                c->kweight[i1 + (long)n1h * (i2 + (long)n[1] * i3)] = ((double)sf * (double)sf) / (double)cnt;
            }
    free(seen);
}

void orc_symmetrize(orc_ctx *c, double *f)
{
    if (c->nops <= 0) return;
    const int *n = c->sys.n;
    const long nr = c->nr;
    double *acc = malloc(sizeof(double) * nr);
    for (int i3 = 0; i3 < n[2]; i3++)
        for (int i2 = 0; i2 < n[1]; i2++)
            for (int i1 = 0; i1 < n[0]; i1++) {
                double s = 0;
                int idx[3] = {i1, i2, i3};
                for (int k = 0; k < c->nops; k++) {
                    const int *M = c->symM + 9 * k, *t = c->symt + 3 * k;
                    int j[3];
                    for (int a = 0; a < 3; a++) {
                        long v = t[a];
                        for (int b = 0; b < 3; b++) v += (long)M[3 * a + b] * idx[b];
                        v %= n[a];
                        if (v < 0) v += n[a];
                        j[a] = (int)v;
                    }
                    s += f[j[0] + (long)n[0] * (j[1] + (long)n[1] * j[2])];
                }
                acc[i1 + (long)n[0] * (i2 + (long)n[1] * i3)] = s / c->nops;
            }
    memcpy(f, acc, sizeof(double) * nr);
    free(acc);
}

/* New cell: G_basis and dGG (the caller runs make_unit_cell) and rebuild k^2
 * (src/iterate_mod.fp.f90:1453-1459 does make_unit_cell + make_ksq). */
void orc_set_cell(orc_ctx *c, const double Gb[3][3], int ncp, const double dGG[][3][3])
{
    memcpy(c->sys.G_basis, Gb, sizeof(double) * 9);
    c->sys.n_cell_param = ncp;
    for (int k = 0; k < ncp; k++) memcpy(c->sys.dGG[k], dGG[k], sizeof(double) * 9);
    orc_make_ksq(c->sys.dim, c->sys.n, c->sys.G_basis, c->ksq, c->gbz);
}

void orc_get_ksq(orc_ctx *c, double *ksq) { memcpy(ksq, c->ksq, sizeof(double) * c->nk); }

/* mu_phi_chain / mu_phi_solvent (src/scf_mod.fp.f90:768-820) */
static void mu_phi(orc_ctx *c)
{
    orc_system *s = &c->sys;
    for (int i = 0; i < s->n_chain; i++) {
        if (s->ensemble == 0) s->mu_chain[i] = log(s->phi_chain[i] / c->qout[i]);
        else s->phi_chain[i] = c->qout[i] * exp(s->mu_chain[i]);
    }
    for (int i = 0; i < s->n_solvent; i++) {
        if (s->ensemble == 0) s->mu_solvent[i] = log(s->phi_solvent[i] / c->qsolv[i]);
        else s->phi_solvent[i] = c->qsolv[i] * exp(s->mu_solvent[i]);
    }
}

/* density() on grid fields (src/scf_mod.fp.f90:144-229 between the basis
 * transforms; for fields of the space-group basis the basis projection of
 * the result is the identity).  omega, rho: [n_monomer][nr]. */
int orc_density(orc_ctx *c, const double *omega, double *rho, double *qout, double *qsolv)
{
    orc_system *s = &c->sys;
    const long nr = c->nr;
    for (int i = 0; i < s->n_chain; i++) {
        chain_density(&c->st, s, i, &c->ch[i], c->ksq, omega);
        c->qout[i] = c->ch[i].bigQ;
    }
    for (long r = 0; r < nr * s->n_monomer; r++) rho[r] = 0.0;
    /* solvent_density (src/scf_mod.fp.f90:251-295) */
    for (int i = 0; i < s->n_solvent; i++) {
        int a = s->solvent_monomer[i];
        double v = s->solvent_size[i];
        const double *w = omega + (long)a * nr;
        double q = 0;
        for (long r = 0; r < nr; r++) q += exp((-v) * w[r]);
        q = q / (double)nr;
        c->qsolv[i] = q;
        if (s->ensemble == 1) s->phi_solvent[i] = q * exp(s->mu_solvent[i]);
        for (long r = 0; r < nr; r++) rho[(long)a * nr + r] += s->phi_solvent[i] * exp((-v) * w[r]) / q;
    }
    if (s->ensemble == 1) mu_phi(c);
    for (int i = 0; i < s->n_chain; i++)
        for (int b = 0; b < s->n_block[i]; b++) {
            int a = s->block_monomer[i][b];
            const double *cr = c->ch[i].rho + (long)b * nr;
            for (long r = 0; r < nr; r++) rho[(long)a * nr + r] = rho[(long)a * nr + r] + s->phi_chain[i] * cr[r];
        }
    if (qout) for (int i = 0; i < s->n_chain; i++) qout[i] = c->qout[i];
    if (qsolv) for (int i = 0; i < s->n_solvent; i++) qsolv[i] = c->qsolv[i];
    return 0;
}

/* Access to the stored propagators of chain ic (after orc_density). */
int orc_chain_slices(orc_ctx *c, int ic) { return c->ch[ic].ns; }
void orc_get_q(orc_ctx *c, int ic, double *qf, double *qr)
{
    long bytes = sizeof(double) * c->nr * c->ch[ic].ns;
    if (qf) memcpy(qf, c->ch[ic].qf, bytes);
    if (qr) memcpy(qr, c->ch[ic].qr, bytes);
}

/* scf_stress (src/scf_mod.fp.f90:451-550).  The star sum
 *   sum_star qf_basis*qr_basis*dGsq   (with basis coefficients from one
 * representative wave, kgrid_to_basis src/grid_basis_mod.f90:146-200)
 * equals, for fields of an orthonormal symmetry-adapted basis, the sum over
 * every wave of the FFT grid of Re(qf^(G) conj(qr^(G))) * dGsq(G), with
 * dGsq(G) = Gbz^T dGG Gbz (src/basis_mod.f90:1993-2014).  The half spectrum
 * counts interior kx planes twice. */
int orc_stress(orc_ctx *c, double *stress)
{
    orc_system *s = &c->sys;
    const long nr = c->nr, nk = c->nk;
    const int n1 = s->n[0], n1h = n1 / 2 + 1;
    const double rn = (double)nr;
    const double normal = rn * rn * 3.0 * 6.0;
    const int ncp = s->n_cell_param;
    cplx *kf = malloc(sizeof(cplx) * nk), *kr = malloc(sizeof(cplx) * nk);
    double *dgsq = malloc(sizeof(double) * nk * (ncp > 0 ? ncp : 1));
    double *wk = malloc(sizeof(double) * nk);
    for (long k = 0; k < nk; k++) {
        int i1 = (int)(k % n1h);
        wk[k] = (i1 == 0 || (n1 % 2 == 0 && i1 == n1 / 2)) ? 1.0 : 2.0;
        if (c->kweight) wk[k] *= c->kweight[k];
        const int *G = c->gbz + 3 * k;
        for (int b = 0; b < ncp; b++) {
            double v = 0;
            for (int j = 0; j < s->dim; j++)
                for (int l = 0; l < s->dim; l++) v += (double)G[j] * (double)G[l] * s->dGG[b][j][l];
            dgsq[k * ncp + b] = v;
        }
    }
    for (int b = 0; b < ncp; b++) stress[b] = 0.0;
    for (int ic = 0; ic < s->n_chain; ic++) {
        chain_work *ch = &c->ch[ic];
        double dQ[ORC_MAXCP] = {0};
        for (int ib = 0; ib < ch->nblk; ib++) {
            int mon = s->block_monomer[ic][ib];
            double bk = s->kuhn[mon];
            double ds0 = ch->block_ds[ib];
            int ibgn = ch->block_bgn[ib], iend = ch->block_bgn[ib + 1];
            for (int i = ibgn; i <= iend; i++) {
                fft3d_r2c(&c->st.f, ch->qf + (long)(i - 1) * nr, kf);
                fft3d_r2c(&c->st.f, ch->qr + (long)(i - 1) * nr, kr);
                double ds = ds0;
                if (i != ibgn && i != iend) ds = (i % 2 == 0) ? 4.0 * ds0 : 2.0 * ds0;
                for (int b = 0; b < ncp; b++) {
                    double inc = 0;
                    for (long k = 0; k < nk; k++)
                        inc += wk[k] * creal(kf[k] * conj(kr[k])) * dgsq[k * ncp + b];
                    inc = inc * (bk * bk) * ds / normal;
                    dQ[b] = dQ[b] - inc;
                }
            }
        }
        for (int b = 0; b < ncp; b++) {
            if (s->ensemble == 0)
                stress[b] = stress[b] - (dQ[b] / ch->bigQ) * s->phi_chain[ic] / ch->length;
            else
                stress[b] = stress[b] - (dQ[b] / ch->bigQ) * exp(s->mu_chain[ic]) * ch->bigQ / ch->length;
        }
    }
    free(kf); free(kr); free(dgsq); free(wk);
    return 0;
}

/* free_energy (src/scf_mod.fp.f90:834-886) with star sums written as grid
 * averages (Parseval for an orthonormal basis).  Uses mu/phi from the last
 * density call.  out[0]=f_Helmholtz, out[1]=pressure. */
int orc_free_energy(orc_ctx *c, const double *omega, const double *rho, double *out)
{
    orc_system *s = &c->sys;
    const long nr = c->nr;
    mu_phi(c);
    double f = 0;
    for (int i = 0; i < s->n_chain; i++) {
        double L = 0;
        for (int b = 0; b < s->n_block[i]; b++) L += s->block_length[i][b];
        if (s->phi_chain[i] > 1.0e-8) f = f + s->phi_chain[i] * (s->mu_chain[i] - 1.0) / L;
    }
    for (int i = 0; i < s->n_solvent; i++)
        if (s->phi_solvent[i] > 1.0e-8) f = f + s->phi_solvent[i] * (s->mu_solvent[i] - 1.0) / s->solvent_size[i];
    double acc = 0;
    if (!c->kweight) {
        for (long r = 0; r < nr; r++) {
            double t = 0;
            for (int a = 0; a < s->n_monomer; a++) {
                for (int b = a + 1; b < s->n_monomer; b++) t += rho[(long)a * nr + r] * s->chi[a][b] * rho[(long)b * nr + r];
                t -= omega[(long)a * nr + r] * rho[(long)a * nr + r];
            }
            acc += t;
        }
        f += acc / (double)nr;
    } else {
        /* star sums of src/scf_mod.fp.f90:861-869 with the star weights */
        const long nk = c->nk;
        const int M = s->n_monomer, n1 = s->n[0], n1h = n1 / 2 + 1;
        cplx *R = malloc(sizeof(cplx) * nk * M), *W = malloc(sizeof(cplx) * nk * M);
        for (int a = 0; a < M; a++) {
            fft3d_r2c(&c->st.f, rho + (long)a * nr, R + (long)a * nk);
            fft3d_r2c(&c->st.f, omega + (long)a * nr, W + (long)a * nk);
        }
        for (long k = 0; k < nk; k++) {
            int i1 = (int)(k % n1h);
            double w = (i1 == 0 || (n1 % 2 == 0 && i1 == n1 / 2)) ? 1.0 : 2.0;
            double t = 0;
            for (int a = 0; a < M; a++) {
                for (int b = a + 1; b < M; b++) t += s->chi[a][b] * creal(R[a * nk + k] * conj(R[b * nk + k]));
                t -= creal(W[a * nk + k] * conj(R[a * nk + k]));
            }
            acc += w * c->kweight[k] * t;
        }
        f += acc / ((double)nr * (double)nr);
        free(R); free(W);
    }
    double p = -f;
    for (int i = 0; i < s->n_chain; i++) {
        double L = 0;
        for (int b = 0; b < s->n_block[i]; b++) L += s->block_length[i][b];
        if (s->phi_chain[i] > 1.0e-8) p = p + s->mu_chain[i] * s->phi_chain[i] / L;
    }
    for (int i = 0; i < s->n_solvent; i++)
        if (s->phi_solvent[i] > 1.0e-8) p = p + s->mu_solvent[i] * s->phi_solvent[i] / s->solvent_size[i];
    out[0] = f;
    out[1] = p;
    return 0;
}

void orc_get_mu_phi(orc_ctx *c, double *mu_chain, double *phi_chain)
{
    for (int i = 0; i < c->sys.n_chain; i++) { mu_chain[i] = c->sys.mu_chain[i]; phi_chain[i] = c->sys.phi_chain[i]; }
}

/* free_energy_FH (src/scf_mod.fp.f90:903-941) */
double orc_free_energy_FH(const orc_system *s)
{
    double f = 0, rho[ORC_MAXM] = {0};
    for (int i = 0; i < s->n_chain; i++) {
        double L = 0;
        for (int b = 0; b < s->n_block[i]; b++) L += s->block_length[i][b];
        if (s->phi_chain[i] > 1.0e-8) f = f + (s->phi_chain[i] / L) * (log(s->phi_chain[i]) - 1);
        for (int b = 0; b < s->n_block[i]; b++)
            rho[s->block_monomer[i][b]] += s->phi_chain[i] * s->block_length[i][b] / L;
    }
    for (int i = 0; i < s->n_solvent; i++) {
        if (s->phi_solvent[i] > 1.0e-8) f = f + (s->phi_solvent[i] / s->solvent_size[i]) * (log(s->phi_solvent[i]) - 1);
        rho[s->solvent_monomer[i]] += s->phi_solvent[i];
    }
    for (int i = 0; i < s->n_monomer - 1; i++)
        for (int j = i + 1; j < s->n_monomer; j++) f = f + s->chi[i][j] * rho[i] * rho[j];
    return f;
}

/* set_omega_uniform (src/scf_mod.fp.f90:724-750): the k=0 component of
 * omega_alpha is sum_beta chi(alpha,beta) phi_mon(beta). */
void orc_omega_uniform(const orc_system *s, double *w0)
{
    double phi_mon[ORC_MAXM] = {0};
    for (int i = 0; i < s->n_chain; i++) {
        double L = 0;
        for (int b = 0; b < s->n_block[i]; b++) L += s->block_length[i][b];
        for (int b = 0; b < s->n_block[i]; b++)
            phi_mon[s->block_monomer[i][b]] += s->phi_chain[i] * s->block_length[i][b] / L;
    }
    for (int i = 0; i < s->n_solvent; i++) phi_mon[s->solvent_monomer[i]] += s->phi_solvent[i];
    for (int a = 0; a < s->n_monomer; a++) {
        w0[a] = 0;
        for (int b = 0; b < s->n_monomer; b++) w0[a] = w0[a] + s->chi[a][b] * phi_mon[b];
    }
}

/* Anderson-mixing deviation (src/iterate_mod.fp.f90:1171-1190) on grid
 * fields, uniform (k=0) component removed: dev[a] = chi.rho + <omega
 * combination>/N_monomer - omega_a.  Returns max |dev| over the grid. */
double orc_am_deviation(const orc_system *s, long nr, const double *omega, const double *rho, double *dev)
{
    const int M = s->n_monomer;
    double emax = 0;
    for (int a = 0; a < M; a++) {
        double mean = 0;
        for (long r = 0; r < nr; r++) {
            double d = 0;
            for (int b = 0; b < M; b++) d += s->chi[b][a] * rho[(long)b * nr + r];
            double sw = 0;
            for (int b = 0; b < M; b++) sw += omega[(long)b * nr + r];
            if (M == 3)
                sw += s->chi[0][1] * rho[2 * nr + r] + s->chi[1][2] * rho[0 * nr + r] + s->chi[0][2] * rho[1 * nr + r];
            d += sw / M - omega[(long)a * nr + r];
            dev[(long)a * nr + r] = d;
            mean += d;
        }
        mean /= (double)nr;
        for (long r = 0; r < nr; r++) {
            dev[(long)a * nr + r] -= mean;
            double v = fabs(dev[(long)a * nr + r]);
            if (v > emax) emax = v;
        }
    }
    return emax;
}

/* ------------------------------------------------------------------ */
/* Unit cell (src/unit_cell_mod.f90:309-664, 723-757)                   */
/* ------------------------------------------------------------------ */

/* Crystal-system codes used by the oracle and the engine's host layer. */
enum {
    ORC_LAMELLAR = 0,
    ORC_SQUARE = 10, ORC_RECTANGULAR = 11, ORC_HEXAGONAL2D = 12, ORC_OBLIQUE = 13,
    ORC_CUBIC = 20, ORC_TETRAGONAL = 21, ORC_ORTHORHOMBIC = 22, ORC_HEXAGONAL3D = 23,
    ORC_MONOCLINIC = 24
};

static void inv3(const double a[3][3], double b[3][3])
{
    double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1])
               - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0])
               + a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    b[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
    b[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    b[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    b[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
    b[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    b[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    b[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
    b[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    b[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
}

/* Returns N_cell_param, or -1 for an unknown system. */
int orc_make_unit_cell(int dim, int system, const double *cp, double G[3][3], double dGG[ORC_MAXCP][3][3])
{
    double R[3][3] = {{0}}, dR[3][3][ORC_MAXCP];
    memset(dR, 0, sizeof(dR));
    int ncp = 0;
    const double twopi = 4.0 * acos(0.0);
    switch (system) {
    case ORC_LAMELLAR:
        ncp = 1; R[0][0] = cp[0]; dR[0][0][0] = 1.0; break;
    case ORC_SQUARE:
        ncp = 1; R[0][0] = cp[0]; R[1][1] = cp[0]; dR[0][0][0] = 1.0; dR[1][1][0] = 1.0; break;
    case ORC_RECTANGULAR:
        ncp = 2; R[0][0] = cp[0]; R[1][1] = cp[1]; dR[0][0][0] = 1.0; dR[1][1][1] = 1.0; break;
    case ORC_HEXAGONAL2D:
        ncp = 1; R[0][0] = cp[0]; R[1][0] = -0.5 * cp[0]; R[1][1] = cp[0] * sqrt(0.75);
        dR[0][0][0] = 1.0; dR[1][0][0] = -0.5; dR[1][1][0] = sqrt(0.75); break;
    case ORC_OBLIQUE:
        /* dR(1,1,1) = a as written in src/unit_cell_mod.f90:630 */
        ncp = 3; R[0][0] = cp[0]; R[1][0] = cp[1] * cos(cp[2]); R[1][1] = cp[1] * sin(cp[2]);
        dR[0][0][0] = cp[0]; dR[1][0][1] = cos(cp[2]); dR[1][1][1] = sin(cp[2]);
        dR[1][0][2] = -cp[1] * sin(cp[2]); dR[1][1][2] = cp[1] * cos(cp[2]); break;
    case ORC_CUBIC:
        ncp = 1; R[0][0] = R[1][1] = R[2][2] = cp[0];
        dR[0][0][0] = dR[1][1][0] = dR[2][2][0] = 1.0; break;
    case ORC_TETRAGONAL:
        ncp = 2; R[0][0] = R[1][1] = cp[0]; R[2][2] = cp[1];
        dR[0][0][0] = dR[1][1][0] = 1.0; dR[2][2][1] = 1.0; break;
    case ORC_ORTHORHOMBIC:
        ncp = 3; R[0][0] = cp[0]; R[1][1] = cp[1]; R[2][2] = cp[2];
        dR[0][0][0] = 1.0; dR[1][1][1] = 1.0; dR[2][2][2] = 1.0; break;
    case ORC_HEXAGONAL3D:
        ncp = 2; R[0][0] = cp[0]; R[1][0] = -0.5 * cp[0]; R[1][1] = cp[0] * sqrt(0.75); R[2][2] = cp[1];
        dR[0][0][0] = 1.0; dR[1][0][0] = -0.5; dR[1][1][0] = sqrt(0.75); dR[2][2][1] = 1.0; break;
    case ORC_MONOCLINIC:
        ncp = 4; R[0][0] = cp[0]; R[1][1] = cp[1]; R[2][0] = cp[2] * cos(cp[3]); R[2][2] = cp[2] * sin(cp[3]);
        dR[0][0][0] = 1.0; dR[1][1][1] = 1.0; dR[2][0][2] = cos(cp[3]); dR[2][2][2] = sin(cp[3]);
        dR[2][0][3] = -cp[2] * sin(cp[3]); dR[2][2][3] = cp[2] * cos(cp[3]); break;
    default:
        return -1;
    }
    /* G = 2 pi inverse(R)^T on the used dim x dim block (src/unit_cell_mod.f90:723-757) */
    double Rl[3][3] = {{0}}, Ri[3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) Rl[i][j] = (i < dim && j < dim) ? R[i][j] : (i == j ? 1.0 : 0.0);
    inv3(Rl, Ri);
    memset(G, 0, sizeof(double) * 9);
    for (int i = 0; i < dim; i++) for (int j = 0; j < dim; j++) G[i][j] = twopi * Ri[j][i];
    double dG[3][3][ORC_MAXCP];
    memset(dG, 0, sizeof(dG));
    for (int k = 0; k < ncp; k++)
        for (int i = 0; i < dim; i++)
            for (int j = 0; j < dim; j++) {
                double s = 0;
                for (int l = 0; l < dim; l++)
                    for (int m = 0; m < dim; m++) s = s - G[i][l] * dR[m][l][k] * G[m][j];
                dG[i][j][k] = s / twopi;
            }
    memset(dGG, 0, sizeof(double) * 9 * ORC_MAXCP);
    for (int k = 0; k < ncp; k++)
        for (int i = 0; i < dim; i++)
            for (int j = 0; j < dim; j++) {
                double s = 0;
                for (int l = 0; l < dim; l++) s = s + G[i][l] * dG[j][l][k] + G[j][l] * dG[i][l][k];
                dGG[k][i][j] = s;
            }
    return ncp;
}

/* ------------------------------------------------------------------ */
/* Anderson mixing (src/iterate_mod.fp.f90:1042-1490) on grid fields    */
/* ------------------------------------------------------------------ */

typedef struct {
    int max_itr;
    int n_hist;
    int domain;
    int crystal_system;
    int verbose;
    double error_max;
} orc_am_param;

typedef struct {
    int itr;
    int converged;
    double error;
    double f_helmholtz;
    double pressure;
    double stress[ORC_MAXCP];
    double cell_param[ORC_MAXCP];
    double q[ORC_MAXC];
    double mu_chain[ORC_MAXC];
} orc_am_result;

/* Solve U x = v by Gaussian elimination with partial pivoting; the
 * reference inverts U with dgetrf/dgetri and multiplies (same algebra). */
static int solve_dense(int n, double *U, double *v)
{
    for (int c = 0; c < n; c++) {
        int p = c;
        for (int r = c + 1; r < n; r++) if (fabs(U[r * n + c]) > fabs(U[p * n + c])) p = r;
        if (U[p * n + c] == 0.0) return -1;
        if (p != c) {
            for (int k = 0; k < n; k++) { double t = U[c * n + k]; U[c * n + k] = U[p * n + k]; U[p * n + k] = t; }
            double t = v[c]; v[c] = v[p]; v[p] = t;
        }
        for (int r = c + 1; r < n; r++) {
            double f = U[r * n + c] / U[c * n + c];
            for (int k = c; k < n; k++) U[r * n + k] -= f * U[c * n + k];
            v[r] -= f * v[c];
        }
    }
    for (int r = n - 1; r >= 0; r--) {
        double s = v[r];
        for (int k = r + 1; k < n; k++) s -= U[r * n + k] * v[k];
        v[r] = s / U[r * n + r];
    }
    return 0;
}

/* omega: [n_monomer][nr] in/out; cell_param in/out (used when domain). */
int orc_iterate_am(orc_ctx *c, double *omega, double *cell_param, const orc_am_param *prm,
                   double *rho, orc_am_result *res)
{
    orc_system *s = &c->sys;
    const long nr = c->nr;
    const int M = s->n_monomer;
    const long fl = (long)M * nr;
    const int H = prm->n_hist;
    const int ncp = prm->domain ? s->n_cell_param : 0;
    double *dev = calloc((size_t)(H + 1) * fl, sizeof(double));
    double *omh = calloc((size_t)(H + 1) * fl, sizeof(double));
    double devcp[64][ORC_MAXCP], cph[64][ORC_MAXCP];
    double *U = malloc(sizeof(double) * H * H), *V = malloc(sizeof(double) * H);
    double stress[ORC_MAXCP] = {0};
    double fe[2];
    memset(devcp, 0, sizeof(devcp)); memset(cph, 0, sizeof(cph));
    double qo[ORC_MAXC], qs[ORC_MAXS];

    for (int a = 0; a < M; a++) orc_symmetrize(c, omega + (long)a * nr);
    orc_density(c, omega, rho, qo, qs);
    mu_phi(c);
    if (s->ensemble == 0) {
        double w0[ORC_MAXM];
        orc_omega_uniform(s, w0);
        for (int a = 0; a < M; a++) {
            double m = 0;
            for (long r = 0; r < nr; r++) m += omega[a * nr + r];
            m /= (double)nr;
            for (long r = 0; r < nr; r++) omega[a * nr + r] += w0[a] - m;
        }
    }
    memcpy(omh, omega, sizeof(double) * fl);
    for (int k = 0; k < ncp; k++) cph[0][k] = cell_param[k];

    int itr = 0, converged = 0;
    double error = 0;
    const double large = 100.0;
    for (;;) {
        itr++;
        int itr_prev;
        double lam;
        if (itr < H + 1) { itr_prev = itr - 1; lam = 1.0 - pow(0.9, itr); }
        else { lam = 1.0; itr_prev = H; }

        orc_density(c, omega, rho, qo, qs);
        if (prm->domain) orc_stress(c, stress);
        mu_phi(c);
        orc_free_energy(c, omega, rho, fe);

        double *dcur = dev + (long)itr_prev * fl;
        double e1 = orc_am_deviation(s, nr, omega, rho, dcur);
        double e2 = 0;
        for (int k = 0; k < ncp; k++) { devcp[itr_prev][k] = -stress[k]; if (fabs(stress[k]) > e2) e2 = fabs(stress[k]); }
        error = e1 > e2 ? e1 : e2;
        if (prm->verbose) {
            fprintf(stderr, "itr %4d error %.3e f %.12f", itr, error, fe[0]);
            for (int k = 0; k < ncp; k++) fprintf(stderr, " cell %.10f stress %.3e", cell_param[k], stress[k]);
            fprintf(stderr, "\n");
        }
        if (error < prm->error_max) { converged = 1; break; }
        if (itr > prm->max_itr) break;
        if (error > 100.0 * large) break;

        if (itr == 1) {
            for (long r = 0; r < fl; r++) omega[r] = omega[r] + lam * dcur[r];
            for (int k = 0; k < ncp; k++) cell_param[k] = cell_param[k] + lam * devcp[0][k];
        } else {
            int n = itr_prev;
            for (int m = 0; m < n; m++) {
                const double *dm = dev + (long)(itr_prev - 1 - m) * fl;
                for (int nn = m; nn < n; nn++) {
                    const double *dn = dev + (long)(itr_prev - 1 - nn) * fl;
                    double u = 0;
                    for (long r = 0; r < fl; r++) u += (dcur[r] - dm[r]) * (dcur[r] - dn[r]);
                    u /= (double)nr;
                    for (int k = 0; k < ncp; k++)
                        u += (devcp[itr_prev][k] - devcp[itr_prev - 1 - m][k]) * (devcp[itr_prev][k] - devcp[itr_prev - 1 - nn][k]);
                    U[m * n + nn] = u; U[nn * n + m] = u;
                }
                double v = 0;
                for (long r = 0; r < fl; r++) v += (dcur[r] - dm[r]) * dcur[r];
                v /= (double)nr;
                for (int k = 0; k < ncp; k++) v += (devcp[itr_prev][k] - devcp[itr_prev - 1 - m][k]) * devcp[itr_prev][k];
                V[m] = v;
            }
            if (solve_dense(n, U, V) != 0) { error = INFINITY; break; }
            const double *wcur = omh + (long)itr_prev * fl;
            for (long r = 0; r < fl; r++) {
                double ww = omega[r], dd = dcur[r];
                for (int nn = 0; nn < n; nn++) {
                    ww += V[nn] * (omh[(long)(itr_prev - 1 - nn) * fl + r] - wcur[r]);
                    dd += V[nn] * (dev[(long)(itr_prev - 1 - nn) * fl + r] - dcur[r]);
                }
                omega[r] = ww + lam * dd;
            }
            for (int k = 0; k < ncp; k++) {
                double ww = cell_param[k], dd = devcp[itr_prev][k];
                for (int nn = 0; nn < n; nn++) {
                    ww += V[nn] * (cph[itr_prev - 1 - nn][k] - cph[itr_prev][k]);
                    dd += V[nn] * (devcp[itr_prev - 1 - nn][k] - devcp[itr_prev][k]);
                }
                cell_param[k] = ww + lam * dd;
            }
        }
        for (int a = 0; a < M; a++) orc_symmetrize(c, omega + (long)a * nr);
        if (itr < H + 1) {
            memcpy(omh + (long)itr * fl, omega, sizeof(double) * fl);
            for (int k = 0; k < ncp; k++) cph[itr][k] = cell_param[k];
        } else {
            memmove(dev, dev + fl, sizeof(double) * fl * H);
            memmove(omh, omh + fl, sizeof(double) * fl * H);
            memcpy(omh + (long)H * fl, omega, sizeof(double) * fl);
            for (int h = 0; h < H; h++) for (int k = 0; k < ncp; k++) { devcp[h][k] = devcp[h + 1][k]; cph[h][k] = cph[h + 1][k]; }
            for (int k = 0; k < ncp; k++) cph[H][k] = cell_param[k];
        }
        if (prm->domain) {
            double G[3][3], dGG[ORC_MAXCP][3][3];
            int nc = orc_make_unit_cell(s->dim, prm->crystal_system, cell_param, G, dGG);
            orc_set_cell(c, G, nc, dGG);
        }
    }
    if (!prm->domain) orc_stress(c, stress);
    res->itr = itr;
    res->converged = converged;
    res->error = error;
    res->f_helmholtz = fe[0];
    res->pressure = fe[1];
    for (int k = 0; k < s->n_cell_param; k++) { res->stress[k] = stress[k]; res->cell_param[k] = cell_param[k]; }
    for (int i = 0; i < s->n_chain; i++) { res->q[i] = qo[i]; res->mu_chain[i] = s->mu_chain[i]; }
    free(dev); free(omh); free(U); free(V);
    return converged ? 0 : 1;
}

/* ------------------------------------------------------------------ */
/* Batch helper for the CPU baseline: n_inst independent density        */
/* evaluations of one system, spread over POSIX threads (one context    */
/* per thread, instances handed out round-robin).                       */
/* ------------------------------------------------------------------ */
typedef struct {
    const orc_system *sys;
    int n_inst, nthreads, tid;
    const double *omega;
    double *rho_out;
} batch_arg;

static void *batch_worker(void *p)
{
    batch_arg *a = (batch_arg *)p;
    orc_ctx *c = orc_create(a->sys);
    long fl = (long)a->sys->n_monomer * c->nr;
    double *rho = malloc(sizeof(double) * fl);
    for (int i = a->tid; i < a->n_inst; i += a->nthreads) {
        orc_density(c, a->omega + (long)i * fl, rho, NULL, NULL);
        if (a->rho_out) memcpy(a->rho_out + (long)i * fl, rho, sizeof(double) * fl);
    }
    free(rho);
    orc_destroy(c);
    return NULL;
}

int orc_density_batch(const orc_system *sys, int n_inst, const double *omega, double *rho_out, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    batch_arg args[256];
    for (int t = 0; t < nthreads; t++) {
        args[t].sys = sys; args[t].n_inst = n_inst; args[t].nthreads = nthreads; args[t].tid = t;
        args[t].omega = omega; args[t].rho_out = rho_out;
        if (pthread_create(&th[t], NULL, batch_worker, &args[t]) != 0) return -1;
    }
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    return 0;
}
