/*
 * bec_oracle.c -- CPU FP64 oracle (test infrastructure; see bec_oracle.h).
 *
 * Restates programs/bec_wigner_3d.cuda of the reference in double precision:
 *   units ............ wigner.cpp:119-176 (fillDerivedParameters)
 *   k table .......... wigner_kernel.cu:15-55 (getK, initWaveVectors)
 *   potential ........ wigner_kernel.cu:99-113
 *   ground state ..... wigner.cu:84-175 with kernels wigner_kernel.cu:116-181, :232-274
 *   ensemble init .... wigner.cu:202-227, wigner_kernel.cu:295-317
 *   split step ....... wigner.cu:178-199, wigner_kernel.cu:137-151, :184-229
 *   pulses ........... wigner_kernel.cu:320-360
 *   observables ...... wigner.cu:257-303, :363-369, wigner_kernel.cu:283-292
 * The FFT is a radix-2 Cooley-Tukey of this file, standing in for cuFFT with
 * the same conventions (forward e^{-i}, inverse e^{+i}, unnormalised; the
 * reference's "k-space" is INVERSE * 1/cells of x-space, wigner.cu:106-107).
 *
 * Defined here (no reference code exists; the product follows the same
 * definitions): Philox4x32-10 noise, the Wigner loss-noise increment, the 2D
 * transverse renormalisation, the mu/energy/residual measures.
 *
 * Pinned (the reference itself cannot be built here) by known-answer tests in
 * tests/test_oracle.py (the published Random123 Philox vectors among them) and
 * by the reference's own stored GPU output: with the loss rates written in its
 * parameter set (wigner.cpp:74-76) this oracle follows data/gpu_sp_30k.yaml
 * within 0.019 in visibility over all of its 0.6 s (tests/test_golden.py).
 */
#include "bec_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* physical constants of wigner.cpp:121-122 */
static const double HBAR = 1.054571628e-34;
static const double BOHR = 5.2917720859e-11;

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
static int ilog2(int n) { int r = 0; while ((1 << r) < n) r++; return r; }

/* ------------------------------------------------------------------ */
/* parameters: fillDerivedParameters, wigner.cpp:119-176               */
/* ------------------------------------------------------------------ */
int oracle_derive(const bec_params *p, bec_derived *d)
{
    if (!p || !d) return BEC_ERR_INVALID_ARG;
    if (!is_pow2(p->nvx) || !is_pow2(p->nvy) || !is_pow2(p->nvz)) return BEC_ERR_UNSUPPORTED_GRID;
    if (p->nvx < 2 || p->nvz < 2) return BEC_ERR_UNSUPPORTED_GRID;
    if (p->m <= 0 || p->fx <= 0 || p->fz <= 0 || p->N <= 0 || p->ne < 1 || p->itmax < 1)
        return BEC_ERR_INVALID_ARG;
    memset(d, 0, sizeof(*d));
    const double w_rho = 2.0 * M_PI * p->fx;                 /* :125 */
    d->l_rho = sqrt(HBAR / (p->m * w_rho));                  /* :126 */
    d->t_rho = 1.0 / w_rho;                                  /* :127 */
    d->lambda = p->fx / p->fz;                               /* :128 */
    d->nvx = p->nvx; d->nvy = p->nvy; d->nvz = p->nvz;
    d->cells = p->nvx * p->nvy * p->nvz;
    d->dims = (p->nvy == 1) ? 2 : 3;
    d->Va = p->Va; d->Vb = p->Vb;
    d->V = (p->Va + p->Vb) / 2.0;                            /* :137 */
    d->detuning = 2.0 * M_PI * p->detuning / w_rho;          /* :139 */
    /* :141-143 with SI rates (no 1e12 / 1e6 division) */
    d->l111 = p->gamma111 / (pow(d->l_rho, 6) * w_rho);
    d->l12 = p->gamma12 / (pow(d->l_rho, 3) * w_rho);
    d->l22 = p->gamma22 / (pow(d->l_rho, 3) * w_rho);
    d->g11 = 4.0 * M_PI * p->a11 * BOHR / d->l_rho;          /* :145-147 */
    d->g12 = 4.0 * M_PI * p->a12 * BOHR / d->l_rho;
    d->g22 = 4.0 * M_PI * p->a22 * BOHR / d->l_rho;
    d->N = p->N;
    if (d->dims == 3) {
        d->mu = pow(15.0 * d->N * d->g11 / (16.0 * M_PI * d->lambda * sqrt(2.0)), 0.4); /* :150 */
        d->xmax = 1.2 * sqrt(2.0 * d->mu);                   /* :153-155 */
        d->ymax = 1.2 * sqrt(2.0 * d->mu);
        d->zmax = 1.2 * d->lambda * sqrt(2.0 * d->mu);
        d->dx = 2.0 * d->xmax / (d->nvx - 1);                /* :158-160 */
        d->dy = 2.0 * d->ymax / (d->nvy - 1);
        d->dz = 2.0 * d->zmax / (d->nvz - 1);
        d->dkx = M_PI / d->xmax;                             /* :167-169 */
        d->dky = M_PI / d->ymax;
        d->dkz = M_PI / d->zmax;
    } else {
        /* 2D x-z slice: the condensate is frozen in the transverse oscillator
         * ground state |phi(y)|^2 = exp(-y^2/l_y^2)/(sqrt(pi) l_y). Couplings
         * and two-body rates scale by int |phi|^4 dy = 1/(sqrt(2 pi) l_y), the
         * three-body rate by int |phi|^6 dy = 1/(sqrt(3) pi l_y^2). */
        const double ly = sqrt(p->fx / (p->fy > 0 ? p->fy : p->fx));   /* l_y / l_rho */
        const double s2 = 1.0 / (sqrt(2.0 * M_PI) * ly);
        const double s3 = 1.0 / (sqrt(3.0) * M_PI * ly * ly);
        d->g11 *= s2; d->g12 *= s2; d->g22 *= s2;
        d->l12 *= s2; d->l22 *= s2; d->l111 *= s3;
        /* 2D Thomas-Fermi: N = pi lambda mu^2 / g11 */
        d->mu = sqrt(d->N * d->g11 / (M_PI * d->lambda));
        d->xmax = 1.2 * sqrt(2.0 * d->mu);
        d->ymax = 0.0;
        d->zmax = 1.2 * d->lambda * sqrt(2.0 * d->mu);
        d->dx = 2.0 * d->xmax / (d->nvx - 1);
        d->dy = 1.0;
        d->dz = 2.0 * d->zmax / (d->nvz - 1);
        d->dkx = M_PI / d->xmax;
        d->dky = 0.0;
        d->dkz = M_PI / d->zmax;
    }
    d->dV = d->dx * d->dy * d->dz;
    d->itmax = p->itmax;
    d->dt_steady = p->dt_steady / d->t_rho;                  /* :172-174 */
    d->t_equilib = p->t_equilib / d->t_rho;
    d->dt_evo = p->dt_evo / d->t_rho;
    d->ne = p->ne;
    /* equilibration loop of wigner.cu:222: for(t = 0; t <= t_equilib; t += dt_evo) */
    {
        int n = 0;
        double t = 0.0;
        if (d->dt_evo > 0) {
            while (t <= d->t_equilib && n < 100000000) { n++; t += d->dt_evo; }
        } else {
            n = 1;
        }
        d->n_equil_steps = n;
    }
    return BEC_OK;
}

/* ------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11)                    */
/* ------------------------------------------------------------------ */
void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        uint32_t n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* -ln(u1) for u1 = (x + 1) / 2^32, accurate at both ends of (0, 1]. */
static double neg_log_u(uint32_t x)
{
    if (x < 0x80000000u) return -log(((double)x + 1.0) * 0x1p-32);
    return -log1p(-((double)(0xFFFFFFFFu - x)) * 0x1p-32);
}

/* Two standard normals from two uniforms (Box-Muller). */
static void box_muller(uint32_t x1, uint32_t x2, double *n1, double *n2)
{
    double r = sqrt(2.0 * neg_log_u(x1));
    double u2 = (double)x2 * 0x1p-32;
    double ang = 2.0 * M_PI * u2;
    *n1 = r * cos(ang);
    *n2 = r * sin(ang);
}

/* Four standard normals for (seed, traj, step, cell, tag):
 * counter = (cell, step, traj, tag), key = (seed low, seed high). */
void oracle_normals4(uint64_t seed, uint32_t traj, uint32_t step, uint32_t cell, uint32_t tag, double out[4])
{
    uint32_t ctr[4] = {cell, step, traj, tag};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t r[4];
    oracle_philox4x32_10(ctr, key, r);
    box_muller(r[0], r[1], &out[0], &out[1]);
    box_muller(r[2], r[3], &out[2], &out[3]);
}

enum { TAG_INIT = 0, TAG_LOSS = 1 };

/* The loss noise of one cell and step (builder definition; no reference counterpart):
 * one Philox4x32-10 draw, counter (cell, step, traj, 1), its 128 bits cut into six 21-bit
 * fields f0..f5 read as three Box-Muller pairs with u1 = (f + 1/2) / 2^21, u2 = f / 2^21. */
void oracle_loss_normals6(uint64_t seed, uint32_t traj, uint32_t step, uint32_t cell, double out[6])
{
    uint32_t ctr[4] = {cell, step, traj, TAG_LOSS};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t w[4], f[6];
    oracle_philox4x32_10(ctr, key, w);
    f[0] = w[0] & 0x1FFFFFu;
    f[1] = (w[0] >> 21) | ((w[1] & 0x3FFu) << 11);
    f[2] = (w[1] >> 10) & 0x1FFFFFu;
    f[3] = (w[1] >> 31) | ((w[2] & 0xFFFFFu) << 1);
    f[4] = (w[2] >> 20) | ((w[3] & 0x1FFu) << 12);
    f[5] = (w[3] >> 9) & 0x1FFFFFu;
    for (int k = 0; k < 3; k++) {
        double r = sqrt(-2.0 * log(((double)f[2 * k] + 0.5) * 0x1p-21));
        double ang = 2.0 * M_PI * ((double)f[2 * k + 1] * 0x1p-21);
        out[2 * k] = r * cos(ang);
        out[2 * k + 1] = r * sin(ang);
    }
}

/* ------------------------------------------------------------------ */
/* FFT: iterative radix-2, unnormalised                                 */
/* ------------------------------------------------------------------ */
typedef struct fft1d {
    int n, logn;
    cplx *tw;       /* n/2 entries exp(-2 pi i k / n) */
    int *rev;
} fft1d;

static void fft1d_init(fft1d *f, int n)
{
    f->n = n; f->logn = ilog2(n);
    f->tw = (cplx *)malloc(sizeof(cplx) * (n / 2 > 0 ? n / 2 : 1));
    f->rev = (int *)malloc(sizeof(int) * n);
    for (int k = 0; k < n / 2; k++) {
        double a = 2.0 * M_PI * (double)k / (double)n;
        f->tw[k] = cos(a) - I * sin(a);
    }
    for (int i = 0; i < n; i++) {
        int r = 0;
        for (int b = 0; b < f->logn; b++) if (i & (1 << b)) r |= 1 << (f->logn - 1 - b);
        f->rev[i] = r;
    }
}

static void fft1d_free(fft1d *f) { free(f->tw); free(f->rev); }

/* in place on contiguous x[0..n) ; sign -1 forward, +1 inverse */
static void fft1d_run(const fft1d *f, cplx *x, int sign)
{
    const int n = f->n;
    if (n == 1) return;
    for (int i = 0; i < n; i++) {
        int r = f->rev[i];
        if (r > i) { cplx t = x[i]; x[i] = x[r]; x[r] = t; }
    }
    for (int half = 1; half < n; half <<= 1) {
        int step = n / (2 * half);
        for (int g = 0; g < n; g += 2 * half) {
            for (int j = 0; j < half; j++) {
                cplx w = f->tw[j * step];
                if (sign > 0) w = conj(w);
                cplx u = x[g + j];
                cplx t = w * x[g + j + half];
                x[g + j] = u + t;
                x[g + j + half] = u - t;
            }
        }
    }
}

typedef struct fft3d {
    int nx, ny, nz;
    fft1d fx, fy, fz;
    cplx *line;
} fft3d;

static void fft3d_init(fft3d *f, int nx, int ny, int nz)
{
    f->nx = nx; f->ny = ny; f->nz = nz;
    fft1d_init(&f->fx, nx); fft1d_init(&f->fy, ny); fft1d_init(&f->fz, nz);
    int m = nx > ny ? nx : ny; if (nz > m) m = nz;
    f->line = (cplx *)malloc(sizeof(cplx) * m);
}

static void fft3d_free(fft3d *f) { fft1d_free(&f->fx); fft1d_free(&f->fy); fft1d_free(&f->fz); free(f->line); }

/* batchfftExecute3D (batchfft.cu:158-180) computes the separable 3D DFT over
 * (z, y, x); the axis order does not change the result. */
static void fft3d_run(fft3d *f, cplx *a, int sign)
{
    const int nx = f->nx, ny = f->ny, nz = f->nz;
    for (int r = 0; r < ny * nz; r++) fft1d_run(&f->fx, a + (size_t)r * nx, sign);
    if (ny > 1) {
        for (int z = 0; z < nz; z++)
            for (int x = 0; x < nx; x++) {
                cplx *base = a + (size_t)z * nx * ny + x;
                for (int y = 0; y < ny; y++) f->line[y] = base[(size_t)y * nx];
                fft1d_run(&f->fy, f->line, sign);
                for (int y = 0; y < ny; y++) base[(size_t)y * nx] = f->line[y];
            }
    }
    for (int p = 0; p < nx * ny; p++) {
        cplx *base = a + p;
        for (int z = 0; z < nz; z++) f->line[z] = base[(size_t)z * nx * ny];
        fft1d_run(&f->fz, f->line, sign);
        for (int z = 0; z < nz; z++) base[(size_t)z * nx * ny] = f->line[z];
    }
}

int oracle_fft3d(double *data, int nx, int ny, int nz, int sign)
{
    if (!is_pow2(nx) || !is_pow2(ny) || !is_pow2(nz)) return BEC_ERR_UNSUPPORTED_GRID;
    fft3d f;
    fft3d_init(&f, nx, ny, nz);
    fft3d_run(&f, (cplx *)data, sign);
    fft3d_free(&f);
    return BEC_OK;
}

/* ------------------------------------------------------------------ */
/* tables: getK / initWaveVectors (wigner_kernel.cu:15-55), potential   */
/* (wigner_kernel.cu:99-113)                                            */
/* ------------------------------------------------------------------ */
static double getK(int i, double dk, int n) { return (2 * i > n) ? dk * (i - n) : dk * i; }

void oracle_k2_table(const bec_derived *d, double *k2h)
{
    for (int z = 0; z < d->nvz; z++)
        for (int y = 0; y < d->nvy; y++)
            for (int x = 0; x < d->nvx; x++) {
                double kx = getK(x, d->dkx, d->nvx);
                double ky = (d->nvy > 1) ? getK(y, d->dky, d->nvy) : 0.0;
                double kz = getK(z, d->dkz, d->nvz);
                k2h[((size_t)z * d->nvy + y) * d->nvx + x] = (kx * kx + ky * ky + kz * kz) / 2.0;
            }
}

void oracle_potential_table(const bec_derived *d, double *v)
{
    for (int z = 0; z < d->nvz; z++)
        for (int y = 0; y < d->nvy; y++)
            for (int x = 0; x < d->nvx; x++) {
                double xx = -d->xmax + d->dx * x;
                double yy = (d->nvy > 1) ? -d->ymax + d->dy * y : 0.0;
                double zz = -d->zmax + d->dz * z;
                v[((size_t)z * d->nvy + y) * d->nvx + x] =
                    (xx * xx + yy * yy + zz * zz / (d->lambda * d->lambda)) / 2.0;
            }
}

/* ------------------------------------------------------------------ */
/* ground state: calculateSteadyState, wigner.cu:84-175                  */
/* ------------------------------------------------------------------ */
static double norm_x(const cplx *psi, int cells, double dV)
{
    double s = 0.0;
    for (int i = 0; i < cells; i++) s += creal(psi[i]) * creal(psi[i]) + cimag(psi[i]) * cimag(psi[i]);
    return s * dV;
}

/* The reference's energy integral (wigner.cu:38-67 with
 * wigner_kernel.cu:232-238, :250-258): sum over cells of
 * n (V + g11 n / 2) + Re(psi(x_i) * psik(k_i) * k_i^2/2), times dV, where
 * psik = INVERSE(psi)/cells. It pairs x- and k-space values of the same
 * index without a conjugate; it only gates the reference's stopping rule. */
static double reference_energy(const cplx *psi, cplx *tmp, fft3d *f, const double *V,
                               const double *k2h, const bec_derived *d)
{
    const int cells = d->cells;
    memcpy(tmp, psi, sizeof(cplx) * cells);
    fft3d_run(f, tmp, +1);
    for (int i = 0; i < cells; i++) tmp[i] /= (double)cells;
    double s = 0.0;
    for (int i = 0; i < cells; i++) {
        double n = creal(psi[i]) * creal(psi[i]) + cimag(psi[i]) * cimag(psi[i]);
        double r = n * (V[i] + d->g11 * n / 2.0);
        cplx t = psi[i] * (tmp[i] * k2h[i]);
        s += r + creal(t);
    }
    return s * d->dV;
}

/* mu, energy per particle and residual ||H psi - mu psi|| / ||psi|| with
 * Parseval kinetic sums: sum_x |psi|^2 = cells * sum_k |psik|^2. */
static void gs_measures(const cplx *psi, cplx *tmp, cplx *tmp2, fft3d *f, const double *V,
                        const double *k2h, const bec_derived *d,
                        double *mu, double *energy, double *residual, double *Nout)
{
    const int cells = d->cells;
    memcpy(tmp, psi, sizeof(cplx) * cells);
    fft3d_run(f, tmp, +1);
    for (int i = 0; i < cells; i++) tmp[i] /= (double)cells;      /* psik */
    double ekin = 0.0, epot = 0.0, eint = 0.0, N = 0.0;
    for (int i = 0; i < cells; i++) {
        double nk = creal(tmp[i]) * creal(tmp[i]) + cimag(tmp[i]) * cimag(tmp[i]);
        ekin += nk * k2h[i];
        double n = creal(psi[i]) * creal(psi[i]) + cimag(psi[i]) * cimag(psi[i]);
        epot += n * V[i];
        eint += n * n;
        N += n;
    }
    ekin *= (double)cells * d->dV;
    epot *= d->dV;
    eint *= d->g11 * d->dV;
    N *= d->dV;
    double m = (ekin + epot + eint) / N;
    /* H psi = FORWARD(psik * k^2/2) + (V + g11 n) psi */
    for (int i = 0; i < cells; i++) tmp2[i] = tmp[i] * k2h[i];
    fft3d_run(f, tmp2, -1);
    double r2 = 0.0, p2 = 0.0;
    for (int i = 0; i < cells; i++) {
        double n = creal(psi[i]) * creal(psi[i]) + cimag(psi[i]) * cimag(psi[i]);
        cplx h = tmp2[i] + (V[i] + d->g11 * n) * psi[i] - m * psi[i];
        r2 += creal(h) * creal(h) + cimag(h) * cimag(h);
        p2 += n;
    }
    if (mu) *mu = m;
    if (energy) *energy = (ekin + epot + 0.5 * eint) / N;
    if (residual) *residual = sqrt(r2 / p2);
    if (Nout) *Nout = N;
}

int oracle_gs_measures(const bec_params *p, const double *psi, double *mu, double *energy,
                       double *residual, double *N)
{
    bec_derived d;
    int st = oracle_derive(p, &d);
    if (st) return st;
    fft3d f; fft3d_init(&f, d.nvx, d.nvy, d.nvz);
    double *V = malloc(sizeof(double) * d.cells), *k2h = malloc(sizeof(double) * d.cells);
    cplx *t1 = malloc(sizeof(cplx) * d.cells), *t2 = malloc(sizeof(cplx) * d.cells);
    oracle_potential_table(&d, V); oracle_k2_table(&d, k2h);
    gs_measures((const cplx *)psi, t1, t2, &f, V, k2h, &d, mu, energy, residual, N);
    free(V); free(k2h); free(t1); free(t2); fft3d_free(&f);
    return BEC_OK;
}

int oracle_ground_state(const bec_params *p, const bec_gs_opts *opts, double *psi_out, bec_gs_report *rep)
{
    bec_derived d;
    int st = oracle_derive(p, &d);
    if (st) return st;
    if (!opts || !psi_out) return BEC_ERR_INVALID_ARG;
    const int cells = d.cells;
    fft3d f; fft3d_init(&f, d.nvx, d.nvy, d.nvz);
    double *V = malloc(sizeof(double) * cells), *k2h = malloc(sizeof(double) * cells);
    double *kprop = malloc(sizeof(double) * cells);
    cplx *a = malloc(sizeof(cplx) * cells), *tmp = malloc(sizeof(cplx) * cells);
    cplx *tmp2 = malloc(sizeof(cplx) * cells);
    cplx *prev = calloc(cells, sizeof(cplx));          /* x-space state at the previous check */
    oracle_potential_table(&d, V); oracle_k2_table(&d, k2h);
    for (int i = 0; i < cells; i++) kprop[i] = exp(-d.dt_steady / 2.0 * k2h[i]);   /* :128-134 */

    /* initial state: fillWithTFGroundState (wigner_kernel.cu:116-125) or warm start */
    if (opts->warm_start) {
        memcpy(a, opts->warm_start, sizeof(cplx) * cells);
    } else {
        for (int i = 0; i < cells; i++) {
            double e = d.mu - V[i];
            a[i] = (e > 0) ? sqrt(e / d.g11) : 0.0;
        }
    }
    /* normalise, then to k-space (wigner.cu:100-107) */
    double N = norm_x(a, cells, d.dV);
    double sc = sqrt(d.N / N);
    for (int i = 0; i < cells; i++) a[i] *= sc;
    fft3d_run(&f, a, +1);
    for (int i = 0; i < cells; i++) a[i] *= 1.0 / cells;

    const int itmax = d.itmax;
    double E = 0.0, mu_prev = 0.0, mu = 0.0, step_res = 0.0;
    int steps = 0, converged = 0, checks = 0;
    const int mu_rule = opts->mode == BEC_GS_MU || opts->mode == BEC_GS_MU_RESIDUAL;
    const double res_tol = opts->res_tol > 0.0 ? opts->res_tol : 10.0 * opts->tol;
    const int maxs = opts->max_steps > 0 ? opts->max_steps : 1;
    const int check = opts->check_every > 0 ? opts->check_every : 1;
    while (steps < maxs) {
        for (int i = 0; i < cells; i++) a[i] *= kprop[i];                  /* :117 */
        fft3d_run(&f, a, -1);                                               /* :121 */
        for (int i = 0; i < cells; i++) {                                   /* :124, kernel :154-181 */
            cplx a0 = a[i], x = a[i];
            double da = 0.0;
            for (int it = 0; it < itmax; it++) {
                double n = creal(x) * creal(x) + cimag(x) * cimag(x);
                da = exp(d.dt_steady / 2.0 * (-V[i] - d.g11 * n));
                x = a0 * da;
            }
            a[i] = x * da;
        }
        fft3d_run(&f, a, +1);                                               /* :129-130 */
        for (int i = 0; i < cells; i++) a[i] *= 1.0 / cells;
        for (int i = 0; i < cells; i++) a[i] *= kprop[i];                  /* :134 */
        fft3d_run(&f, a, -1);                                               /* :140 */
        N = norm_x(a, cells, d.dV);                                         /* :143-145 */
        sc = sqrt(d.N / N);
        for (int i = 0; i < cells; i++) a[i] *= sc;
        steps++;
        int stop = 0;
        if (opts->mode == BEC_GS_REFERENCE_E) {
            double newE = reference_energy(a, tmp, &f, V, k2h, &d);        /* :148 */
            if (fabs((newE - E) / newE) < 0.000001) stop = 1;              /* :155 */
            E = newE;
        } else if (mu_rule && (steps % check) == 0) {
            gs_measures(a, tmp, tmp2, &f, V, k2h, &d, &mu, NULL, NULL, NULL);
            /* fixed-point residual || psi_n - psi_{n-c} || / (c dt mu || psi_n ||) */
            double dd = 0.0, nn = 0.0;
            for (int i = 0; i < cells; i++) {
                const cplx e = a[i] - prev[i];
                dd += creal(e) * creal(e) + cimag(e) * cimag(e);
                nn += creal(a[i]) * creal(a[i]) + cimag(a[i]) * cimag(a[i]);
                prev[i] = a[i];
            }
            const double r = sqrt(dd / nn) / ((double)check * d.dt_steady * fabs(mu));
            if (checks > 0) step_res = r;
            const int mu_ok = mu_prev != 0.0 && fabs((mu - mu_prev) / mu) < opts->tol;
            if (mu_ok && (opts->mode == BEC_GS_MU || (checks > 0 && r < res_tol))) stop = 1;
            mu_prev = mu;
            ++checks;
        }
        fft3d_run(&f, a, +1);                                               /* :151-152 */
        for (int i = 0; i < cells; i++) a[i] *= 1.0 / cells;
        if (stop) { converged = 1; break; }
    }
    fft3d_run(&f, a, -1);                                                   /* :163 */
    memcpy(psi_out, a, sizeof(cplx) * cells);
    if (rep) {
        memset(rep, 0, sizeof(*rep));
        rep->steps = steps;
        rep->converged = converged;
        rep->step_residual = step_res;
        gs_measures(a, tmp, tmp2, &f, V, k2h, &d, &rep->mu, &rep->energy, &rep->residual, &rep->N);
    }
    free(V); free(k2h); free(kprop); free(a); free(tmp); free(tmp2); free(prev); fft3d_free(&f);
    return BEC_OK;
}

/* ------------------------------------------------------------------ */
/* ensembles                                                            */
/* ------------------------------------------------------------------ */
struct oracle_ens {
    bec_params p;
    bec_derived d;
    cplx *a, *b;          /* k-space, ne * cells each (EvolutionState a, b: defines.h:119) */
    double *V, *k2h;
    long long step;       /* steps taken since init (Philox counter) */
    double t;             /* natural time since start_evolution */
    int initialised;
};

oracle_ens *oracle_create(const bec_params *p)
{
    oracle_ens *e = calloc(1, sizeof(*e));
    if (!e) return NULL;
    if (oracle_derive(p, &e->d) != BEC_OK) { free(e); return NULL; }
    e->p = *p;
    size_t n = (size_t)e->d.cells * e->d.ne;
    e->a = calloc(n, sizeof(cplx));
    e->b = calloc(n, sizeof(cplx));
    e->V = malloc(sizeof(double) * e->d.cells);
    e->k2h = malloc(sizeof(double) * e->d.cells);
    oracle_potential_table(&e->d, e->V);
    oracle_k2_table(&e->d, e->k2h);
    return e;
}

void oracle_free(oracle_ens *e)
{
    if (!e) return;
    free(e->a); free(e->b); free(e->V); free(e->k2h); free(e);
}

/* initializeEnsembles (wigner_kernel.cu:295-317) then INVERSE * 1/cells
 * (wigner.cu:216-218). eta has sigma 0.5 per part (wigner.cu:211). */
int oracle_init(oracle_ens *e, const double *psi_gs, const double *noise)
{
    if (!e || !psi_gs) return BEC_ERR_INVALID_ARG;
    const bec_derived *d = &e->d;
    const int cells = d->cells;
    const double coeff = 1.0 / sqrt(d->dV);
    const cplx *gs = (const cplx *)psi_gs;
    const cplx *nz = (const cplx *)noise;
    fft3d f; fft3d_init(&f, d->nvx, d->nvy, d->nvz);
    for (int t = 0; t < d->ne; t++) {
        cplx *a = e->a + (size_t)t * cells, *b = e->b + (size_t)t * cells;
        for (int i = 0; i < cells; i++) {
            cplx ea, eb;
            if (nz) {
                ea = nz[((size_t)t * 2 + 0) * cells + i];
                eb = nz[((size_t)t * 2 + 1) * cells + i];
            } else {
                double r[4];
                oracle_normals4(e->p.seed, (uint32_t)t, 0u, (uint32_t)i, TAG_INIT, r);
                ea = 0.5 * r[0] + I * 0.5 * r[1];
                eb = 0.5 * r[2] + I * 0.5 * r[3];
            }
            a[i] = gs[i] + d->Va * ea * coeff;
            b[i] = d->Vb * eb * coeff;
        }
        fft3d_run(&f, a, +1);
        fft3d_run(&f, b, +1);
        for (int i = 0; i < cells; i++) { a[i] *= 1.0 / cells; b[i] *= 1.0 / cells; }
    }
    fft3d_free(&f);
    e->step = 0;
    e->t = 0.0;
    e->initialised = 1;
    return BEC_OK;
}

static inline cplx cexp_ref(cplx z) { double m = exp(creal(z)); return m * cos(cimag(z)) + I * (m * sin(cimag(z))); }

/* One real-time step of one trajectory: propagate (wigner.cu:178-199). */
static void step_traj(const oracle_ens *e, fft3d *f, cplx *a, cplx *b, int traj, long long step)
{
    const bec_derived *d = &e->d;
    const int cells = d->cells;
    const double dt = d->dt_evo;
    /* propagateKSpaceRealTime (wigner_kernel.cu:137-151): angle +k^2/2 * dt/2 */
    for (int i = 0; i < cells; i++) {
        double ang = e->k2h[i] * dt / 2.0;
        cplx c = cos(ang) + I * sin(ang);
        a[i] *= c; b[i] *= c;
    }
    fft3d_run(f, a, -1);
    fft3d_run(f, b, -1);
    /* propagateXSpaceTwoComponent (wigner_kernel.cu:184-229) */
    const int noise = e->p.loss_noise && (d->l111 > 0 || d->l12 > 0 || d->l22 > 0);
    const double ns = sqrt(dt / (2.0 * d->dV));
    const double c1 = sqrt(d->l111 / 6.0) * 3.0, c2 = sqrt(d->l12 / 2.0), c3 = sqrt(d->l22);
    for (int i = 0; i < cells; i++) {
        const double V = e->V[i];
        cplx a0 = a[i], b0 = b[i], x = a0, y = b0;
        cplx da = 0.0, db = 0.0;
        for (int it = 0; it < d->itmax; it++) {
            double na = creal(x) * creal(x) + cimag(x) * cimag(x);
            double nb = creal(y) * creal(y) + cimag(y) * cimag(y);
            cplx pa = -(d->l111 * na * na + d->l12 * nb) / 2.0 + I * (-(-V - d->g11 * na - d->g12 * nb));
            cplx pb = -(d->l22 * nb + d->l12 * na) / 2.0 +
                      I * (-(-V - d->g22 * nb - d->g12 * na + d->detuning));
            da = cexp_ref(pa * (dt / 2.0));
            db = cexp_ref(pb * (dt / 2.0));
            x = a0 * da;
            y = b0 * db;
        }
        cplx ao = x * da, bo = y * db;
        if (noise) {
            /* Wigner loss noise, Euler-Maruyama at the start of the substep:
             *   da += sqrt(l111/6) 3 conj(a)^2 dW1 + sqrt(l12/2) conj(b) dW2
             *   db += sqrt(l12/2) conj(a) dW2 + sqrt(l22) conj(b) dW3
             * <dW dW*> = dt/dV per channel (diffusion of report.tex:700-720,
             * poster.tex:276-278 with kappa fixed by the drift of :208-215). */
            double r[6];
            oracle_loss_normals6(e->p.seed, (uint32_t)traj, (uint32_t)step, (uint32_t)i, r);
            cplx w1 = ns * (r[0] + I * r[1]);
            cplx w2 = ns * (r[2] + I * r[3]);
            cplx w3 = ns * (r[4] + I * r[5]);
            cplx ca = conj(a0), cb = conj(b0);
            ao += c1 * ca * ca * w1 + c2 * cb * w2;
            bo += c2 * ca * w2 + c3 * cb * w3;
        }
        a[i] = ao; b[i] = bo;
    }
    fft3d_run(f, a, +1);
    fft3d_run(f, b, +1);
    for (int i = 0; i < cells; i++) {      /* multiplyPair (wigner.cu:193), then K/2 (:197) */
        double ang = e->k2h[i] * dt / 2.0;
        cplx c = cos(ang) + I * sin(ang);
        a[i] *= 1.0 / cells; b[i] *= 1.0 / cells;
        a[i] *= c; b[i] *= c;
    }
}

int oracle_evolve(oracle_ens *e, int n_steps, int threads)
{
    if (!e || !e->initialised) return BEC_ERR_STATE;
    if (n_steps <= 0) return BEC_OK;
    const int cells = e->d.cells;
    const int ne = e->d.ne;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (int t = 0; t < ne; t++) {
        fft3d f; fft3d_init(&f, e->d.nvx, e->d.nvy, e->d.nvz);
        cplx *a = e->a + (size_t)t * cells, *b = e->b + (size_t)t * cells;
        for (int s = 0; s < n_steps; s++) step_traj(e, &f, a, b, t, e->step + s);
        fft3d_free(&f);
    }
    (void)threads;
    e->step += n_steps;
    e->t += n_steps * e->d.dt_evo;
    return BEC_OK;
}

/* report.tex rotation matrix; theta = pi/2 is applyHalfPiPulse (wigner_kernel.cu:320-329) */
int oracle_pulse(oracle_ens *e, double theta, double phi)
{
    if (!e || !e->initialised) return BEC_ERR_STATE;
    const double c = cos(theta / 2.0), s = sin(theta / 2.0);
    const cplx m12 = -I * cexp_ref(-I * phi) * s;
    const cplx m21 = -I * cexp_ref(I * phi) * s;
    size_t n = (size_t)e->d.cells * e->d.ne;
    for (size_t i = 0; i < n; i++) {
        cplx a = e->a[i], b = e->b[i];
        e->a[i] = c * a + m12 * b;
        e->b[i] = m21 * a + c * b;
    }
    return BEC_OK;
}

/* Rounds every stored amplitude to FP32 and back (no reference counterpart): a perturbation of FP32
 * rounding size, applied after every step of a second oracle run, shows how far rounding alone moves
 * the trajectories of a configuration. */
int oracle_round_fp32(oracle_ens *e)
{
    if (!e || !e->initialised) return BEC_ERR_STATE;
    size_t n = (size_t)e->d.cells * e->d.ne;
    for (size_t i = 0; i < n; i++) {
        e->a[i] = (double)(float)creal(e->a[i]) + I * (double)(float)cimag(e->a[i]);
        e->b[i] = (double)(float)creal(e->b[i]) + I * (double)(float)cimag(e->b[i]);
    }
    return BEC_OK;
}

/* initEvolution's tail (wigner.cu:222-225): equilibration steps, then pi/2. */
int oracle_start_evolution(oracle_ens *e, int threads)
{
    int st = oracle_evolve(e, e->d.n_equil_steps, threads);
    if (st) return st;
    st = oracle_pulse(e, M_PI / 2.0, 0.0);
    e->t = 0.0;
    return st;
}

/* x-space copy of one trajectory */
static void to_x(const oracle_ens *e, fft3d *f, int t, cplx *xa, cplx *xb)
{
    const int cells = e->d.cells;
    memcpy(xa, e->a + (size_t)t * cells, sizeof(cplx) * cells);
    memcpy(xb, e->b + (size_t)t * cells, sizeof(cplx) * cells);
    fft3d_run(f, xa, -1);
    fft3d_run(f, xb, -1);
}

int oracle_traj_moments(oracle_ens *e, bec_moments *out)
{
    if (!e || !e->initialised || !out) return BEC_ERR_INVALID_ARG;
    const int cells = e->d.cells;
    fft3d f; fft3d_init(&f, e->d.nvx, e->d.nvy, e->d.nvz);
    cplx *xa = malloc(sizeof(cplx) * cells), *xb = malloc(sizeof(cplx) * cells);
    for (int t = 0; t < e->d.ne; t++) {
        to_x(e, &f, t, xa, xb);
        double na = 0, nb = 0;
        cplx s = 0;
        for (int i = 0; i < cells; i++) {
            na += creal(xa[i]) * creal(xa[i]) + cimag(xa[i]) * cimag(xa[i]);
            nb += creal(xb[i]) * creal(xb[i]) + cimag(xb[i]) * cimag(xb[i]);
            s += conj(xa[i]) * xb[i];
        }
        out[t].t = e->t * e->d.t_rho;
        out[t].na = na * e->d.dV;
        out[t].nb = nb * e->d.dV;
        out[t].s_re = creal(s) * e->d.dV;
        out[t].s_im = cimag(s) * e->d.dV;
    }
    free(xa); free(xb); fft3d_free(&f);
    return BEC_OK;
}

int oracle_moments(oracle_ens *e, bec_moments *out)
{
    if (!e || !e->initialised || !out) return BEC_ERR_INVALID_ARG;
    bec_moments *tm = malloc(sizeof(bec_moments) * e->d.ne);
    oracle_traj_moments(e, tm);
    memset(out, 0, sizeof(*out));
    out->t = e->t * e->d.t_rho;
    for (int t = 0; t < e->d.ne; t++) {
        out->na += tm[t].na; out->nb += tm[t].nb;
        out->s_re += tm[t].s_re; out->s_im += tm[t].s_im;
    }
    free(tm);
    return BEC_OK;
}

int oracle_axial(oracle_ens *e, double *out)
{
    if (!e || !e->initialised || !out) return BEC_ERR_INVALID_ARG;
    const bec_derived *d = &e->d;
    const int cells = d->cells, plane = d->nvx * d->nvy;
    fft3d f; fft3d_init(&f, d->nvx, d->nvy, d->nvz);
    cplx *xa = malloc(sizeof(cplx) * cells), *xb = malloc(sizeof(cplx) * cells);
    memset(out, 0, sizeof(double) * 4 * d->nvz);
    for (int t = 0; t < d->ne; t++) {
        to_x(e, &f, t, xa, xb);
        for (int z = 0; z < d->nvz; z++) {
            double na = 0, nb = 0; cplx s = 0;
            for (int i = 0; i < plane; i++) {
                cplx u = xa[(size_t)z * plane + i], v = xb[(size_t)z * plane + i];
                na += creal(u) * creal(u) + cimag(u) * cimag(u);
                nb += creal(v) * creal(v) + cimag(v) * cimag(v);
                s += conj(u) * v;
            }
            out[4 * z + 0] += na * d->dV;
            out[4 * z + 1] += nb * d->dV;
            out[4 * z + 2] += creal(s) * d->dV;
            out[4 * z + 3] += cimag(s) * d->dV;
        }
    }
    free(xa); free(xb); fft3d_free(&f);
    return BEC_OK;
}

int oracle_get_state(oracle_ens *e, int traj, double *ab)
{
    if (!e || !e->initialised || !ab || traj < 0 || traj >= e->d.ne) return BEC_ERR_INVALID_ARG;
    fft3d f; fft3d_init(&f, e->d.nvx, e->d.nvy, e->d.nvz);
    to_x(e, &f, traj, (cplx *)ab, (cplx *)ab + e->d.cells);
    fft3d_free(&f);
    return BEC_OK;
}

int oracle_set_state(oracle_ens *e, int traj, const double *ab)
{
    if (!e || !ab || traj < 0 || traj >= e->d.ne) return BEC_ERR_INVALID_ARG;
    const int cells = e->d.cells;
    fft3d f; fft3d_init(&f, e->d.nvx, e->d.nvy, e->d.nvz);
    cplx *a = e->a + (size_t)traj * cells, *b = e->b + (size_t)traj * cells;
    memcpy(a, ab, sizeof(cplx) * cells);
    memcpy(b, (const cplx *)ab + cells, sizeof(cplx) * cells);
    fft3d_run(&f, a, +1);
    fft3d_run(&f, b, +1);
    for (int i = 0; i < cells; i++) { a[i] *= 1.0 / cells; b[i] *= 1.0 / cells; }
    fft3d_free(&f);
    e->initialised = 1;
    return BEC_OK;
}

long long oracle_step_index(const oracle_ens *e) { return e ? e->step : -1; }
double oracle_time(const oracle_ens *e) { return e ? e->t * e->d.t_rho : 0.0; }

/* halfPiRotate (wigner_kernel.cu:344-360) + density (:283-286) + reduce over the
 * whole ensemble (wigner.cu:259-263); returned sums are multiplied by dV. */
int oracle_ref_rotated_sums(oracle_ens *e, double alpha, double *na_out, double *nb_out)
{
    if (!e || !e->initialised) return BEC_ERR_STATE;
    const bec_derived *d = &e->d;
    const int cells = d->cells;
    const double root2 = sqrt(2.0), ca = cos(alpha), sa = sin(alpha);
    const double sub = d->V / (2.0 * d->dx * d->dy * d->dz);
    fft3d f; fft3d_init(&f, d->nvx, d->nvy, d->nvz);
    cplx *xa = malloc(sizeof(cplx) * cells), *xb = malloc(sizeof(cplx) * cells);
    double sa_sum = 0.0, sb_sum = 0.0;
    for (int t = 0; t < d->ne; t++) {
        to_x(e, &f, t, xa, xb);
        for (int i = 0; i < cells; i++) {
            cplx a0 = xa[i], b0 = xb[i];
            cplx an = (a0 + b0 * (sa - I * ca)) * (1.0 / root2);
            cplx bn = (a0 * (-sa - I * ca) + b0) * (1.0 / root2);
            sa_sum += creal(an) * creal(an) + cimag(an) * cimag(an) - sub;
            sb_sum += creal(bn) * creal(bn) + cimag(bn) * cimag(bn) - sub;
        }
    }
    free(xa); free(xb); fft3d_free(&f);
    *na_out = sa_sum * d->dV;
    *nb_out = sb_sum * d->dV;
    return BEC_OK;
}

/* getVisibility (wigner.cu:257-277): alpha = 0, 0.5, ... < 2 pi */
int oracle_ref_visibility(oracle_ens *e, double *vis)
{
    double mx = 0.0;
    for (double alpha = 0; alpha < 2 * M_PI; alpha += 0.5) {
        double na, nb;
        int st = oracle_ref_rotated_sums(e, alpha, &na, &nb);
        if (st) return st;
        double n1 = fabs(na), n2 = fabs(nb);
        double r = (n1 - n2) / (n1 + n2);
        if (fabs(r) > mx) mx = fabs(r);
    }
    *vis = mx;
    return BEC_OK;
}

/* printComponentRatioAxialProjection (wigner.cu:279-303): (a - b) / (a + b) per z */
int oracle_ref_axial_ratio(oracle_ens *e, double *out)
{
    if (!e || !e->initialised) return BEC_ERR_STATE;
    const bec_derived *d = &e->d;
    const int cells = d->cells, plane = d->nvx * d->nvy;
    const double root2 = sqrt(2.0);
    const double sub = d->V / (2.0 * d->dx * d->dy * d->dz);
    fft3d f; fft3d_init(&f, d->nvx, d->nvy, d->nvz);
    cplx *xa = malloc(sizeof(cplx) * cells), *xb = malloc(sizeof(cplx) * cells);
    double *pa = calloc(d->nvz, sizeof(double)), *pb = calloc(d->nvz, sizeof(double));
    for (int t = 0; t < d->ne; t++) {
        to_x(e, &f, t, xa, xb);
        for (int i = 0; i < cells; i++) {
            cplx a0 = xa[i], b0 = xb[i];
            cplx an = (a0 - I * b0) * (1.0 / root2);
            cplx bn = (-I * a0 + b0) * (1.0 / root2);
            pa[i / plane] += creal(an) * creal(an) + cimag(an) * cimag(an) - sub;
            pb[i / plane] += creal(bn) * creal(bn) + cimag(bn) * cimag(bn) - sub;
        }
    }
    for (int z = 0; z < d->nvz; z++) out[z] = (pa[z] - pb[z]) / (pa[z] + pb[z]);
    free(xa); free(xb); free(pa); free(pb); fft3d_free(&f);
    return BEC_OK;
}
