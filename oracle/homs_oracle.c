/*
 * homs_oracle.c -- CPU FP64 restatement of HighOrderMRISim.jl's BlochHighOrder
 * simulation path.  TEST INFRASTRUCTURE ONLY: this file is the checker that the
 * CUDA engine is compared against (and the timed CPU baseline in bench.py).  The
 * product never links or calls it.
 *
 * Reference semantics followed here (paths inside the HighOrderMRISim.jl tree):
 *   - basis terms and their expression order:
 *       src/simulation/Bloch/BlochHighOrderSimulatitonMethod.jl:54-68
 *   - field selection, "first order replaces nominal gradients", Δw term:
 *       src/simulation/Bloch/BlochHighOrderSimulatitonMethod.jl:70-75
 *   - phase  φ = -2πγ·cumtrapz(Δt, Bz)   (KomaMRICore 0.14 cumtrapz: sequential
 *       cumulative sum of (B[n+1]+B[n])·Δt[n], halved):  ...SimulatonMethod.jl:78
 *   - Mxy = M0·exp(iφ - t'/T2), Mz relaxation over the block, ADC columns
 *       ADC[2:end], signal = transpose(states)·csm:       ...SimulatonMethod.jl:83-92
 *   - excitation loop (start-node values, spinor, relaxation, ADC-during-RF,
 *       ψ framing):                                        ...SimulatonMethod.jl:100-134
 *   - hard-pulse spinor restated in-tree:   src/simulation/kernels/HighOrderGPU.jl:181-192
 *   - block loop, ADC ownership of shared boundary nodes:
 *       src/simulation/SimulatorCore.jl:96-152
 *   - BlochHighOrder mask bits:             src/simulation/BlochHighOrder.jl:21-43
 *
 * Arithmetic is plain IEEE double with no contraction (build with
 * -ffp-contract=off), in the reference's expression order, so the CUDA FP64
 * kernel that follows the same order can agree to ~1e-15.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define OR_HO0 1u
#define OR_HO1 2u
#define OR_HO2 4u
#define OR_HO3 8u
#define OR_DW_EXC 16u
#define OR_DW_PREC 32u

typedef struct or_phantom {
    int64_t ns;
    int32_t nc;
    const double *x, *y, *z, *rho, *T1, *T2, *dw;
    const double *csm; /* interleaved complex, column-major ns x nc: (s,c) at 2*(s + c*ns) */
} or_phantom;

typedef struct or_sequence {
    int64_t nt;
    const double *t, *dt; /* nt, nt-1 */
    const double *gx, *gy, *gz;
    const double *b1; /* interleaved complex, nt */
    const double *df, *psi;
    const uint8_t *adc;
    const double *h[16];
    int32_t nblocks;
    const int64_t *first, *last; /* 0-based inclusive node range per block */
    const uint8_t *exc;          /* 1 = excitation block */
    double gamma;                /* Hz/T */
} or_sequence;

/* Sixteen unnormalised real solid harmonics, CPU expression order
 * (BlochHighOrderSimulatitonMethod.jl:54-68). */
void oracle_basis(double x, double y, double z, double *b)
{
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double r2 = (x2 + y2) + z2;
    b[0] = 1.0;
    b[1] = x;
    b[2] = y;
    b[3] = z;
    b[4] = x * y;
    b[5] = z * y;
    b[6] = 3.0 * z2 - r2;
    b[7] = x * z;
    b[8] = x2 - y2;
    b[9] = (3.0 * y) * x2 - (y2 * y);
    b[10] = (x * z) * y;
    b[11] = (5.0 * z2 - r2) * y;
    b[12] = 5.0 * (z2 * z) - (3.0 * z) * r2;
    b[13] = (5.0 * z2 - r2) * x;
    b[14] = x2 * z - y2 * z;
    b[15] = (x2 * x) - (3.0 * x) * y2;
}

/* Bz at one node, CPU association ((((Bz0+Bz1)+Bz2)+Bz3)+Δw/(2πγ))
 * (BlochHighOrderSimulatitonMethod.jl:70-75). */
static double field_at(const or_sequence *q, const double *b, double dwterm, uint32_t m, int64_t n)
{
    double bz0 = (m & OR_HO0) ? q->h[0][n] : 0.0;
    double bz1;
    if (m & OR_HO1)
        bz1 = (b[1] * q->h[1][n] + b[2] * q->h[2][n]) + b[3] * q->h[3][n];
    else
        bz1 = (b[1] * q->gx[n] + b[2] * q->gy[n]) + b[3] * q->gz[n];
    double bz2 = 0.0, bz3 = 0.0;
    if (m & OR_HO2)
        bz2 = (((b[4] * q->h[4][n] + b[5] * q->h[5][n]) + b[6] * q->h[6][n]) + b[7] * q->h[7][n]) +
              b[8] * q->h[8][n];
    if (m & OR_HO3)
        bz3 = (((((b[9] * q->h[9][n] + b[10] * q->h[10][n]) + b[11] * q->h[11][n]) + b[12] * q->h[12][n]) +
                b[13] * q->h[13][n]) +
               b[14] * q->h[14][n]) +
              b[15] * q->h[15][n];
    double bz = ((bz0 + bz1) + bz2) + bz3;
    if (m & OR_DW_PREC) bz = bz + dwterm;
    return bz;
}

/* Julia complex product (re*re - im*im, re*im + im*re). */
static inline void cmul(double ar, double ai, double br, double bi, double *cr, double *ci)
{
    double r = ar * br - ai * bi;
    double i = ar * bi + ai * br;
    *cr = r;
    *ci = i;
}

/* Number of ADC samples owned by block k: ADC[first+1 .. last]
 * (SimulatorCore.jl:115-116). */
static int64_t block_adc(const or_sequence *q, int32_t k)
{
    int64_t c = 0;
    for (int64_t n = q->first[k] + 1; n <= q->last[k]; ++n) c += q->adc[n] ? 1 : 0;
    return c;
}

int64_t oracle_count_adc(const or_sequence *q)
{
    int64_t c = 0;
    for (int32_t k = 0; k < q->nblocks; ++k) c += block_adc(q, k);
    return c;
}

/* One precession block for spins [s0,s1): run_spin_precession!
 * (BlochHighOrderSimulatitonMethod.jl:43-94).  `acc` accumulates this
 * thread's contribution to the block's signal, (nadc x nc) column-major. */
static void precession_block(const or_phantom *p, const or_sequence *q, uint32_t m, int32_t k, int64_t s0,
                             int64_t s1, double *mxy, double *mz, double *acc, int64_t nadc)
{
    const int64_t f = q->first[k], l = q->last[k];
    const double twopig = 2.0 * M_PI * q->gamma; /* T(2π*γ) */
    const double c2 = -twopig;                   /* T(-2π*γ) */
    for (int64_t s = s0; s < s1; ++s) {
        double b[16];
        oracle_basis(p->x[s], p->y[s], p->z[s], b);
        double dwterm = p->dw[s] / twopig;
        double m0r = mxy[2 * s], m0i = mxy[2 * s + 1];
        double prev = field_at(q, b, dwterm, m, f);
        double cum = 0.0, tp = 0.0;
        double er = m0r, ei = m0i; /* state at the last node */
        int64_t sample = 0;
        for (int64_t n = f; n < l; ++n) {
            double next = field_at(q, b, dwterm, m, n + 1);
            double y = (next + prev) * q->dt[n];
            cum = cum + y;
            tp = tp + q->dt[n];
            int take = q->adc[n + 1] || (n + 1 == l);
            if (take) {
                double phi = c2 * (0.5 * cum);
                double e = exp(0.0 - tp / p->T2[s]);
                double sn = sin(phi), cs = cos(phi);
                double xr, xi;
                cmul(m0r, m0i, e * cs, e * sn, &xr, &xi);
                er = xr;
                ei = xi;
                if (q->adc[n + 1] && nadc > 0) {
                    for (int32_t c = 0; c < p->nc; ++c) {
                        const double *w = p->csm + 2 * (s + (int64_t)c * p->ns);
                        double vr, vi;
                        cmul(xr, xi, w[0], w[1], &vr, &vi);
                        double *o = acc + 2 * (sample + (int64_t)c * nadc);
                        o[0] += vr;
                        o[1] += vi;
                    }
                    sample++;
                }
            }
            prev = next;
        }
        double e1 = exp(-tp / p->T1[s]);
        mxy[2 * s] = er;
        mxy[2 * s + 1] = ei;
        mz[s] = mz[s] * e1 + p->rho[s] * (1.0 - e1);
    }
}

/* One excitation block for spins [s0,s1): run_spin_excitation!
 * (BlochHighOrderSimulatitonMethod.jl:100-134) with the hard-pulse spinor of
 * kernels/HighOrderGPU.jl:181-192. */
static void excitation_block(const or_phantom *p, const or_sequence *q, uint32_t m, int32_t k, int64_t s0,
                             int64_t s1, double *mxy, double *mz, double *acc, int64_t nadc)
{
    const int64_t f = q->first[k], l = q->last[k];
    const double twopig = 2.0 * M_PI * q->gamma;
    const double c2 = -twopig;
    const double eps = 2.220446049250313e-16;
    for (int64_t s = s0; s < s1; ++s) {
        double xr = mxy[2 * s], xi = mxy[2 * s + 1], zz = mz[s];
        /* M.xy .*= cis(-ψ[1]) */
        cmul(xr, xi, cos(-q->psi[f]), sin(-q->psi[f]), &xr, &xi);
        double off = (m & OR_DW_EXC) ? p->dw[s] / twopig : 0.0;
        int64_t sample = 0;
        for (int64_t n = f; n < l; ++n) {
            double dbz = off - q->df[n] / q->gamma;
            double bz = ((q->gx[n] * p->x[s] + q->gy[n] * p->y[s]) + q->gz[n] * p->z[s]) + dbz;
            double b1r = q->b1[2 * n], b1i = q->b1[2 * n + 1];
            double ab1 = hypot(b1r, b1i);
            double B = sqrt(ab1 * ab1 + bz * bz);
            if (B == 0.0) B = eps;
            double phi = c2 * (B * q->dt[n]);
            double sh = sin(phi / 2.0), ch = cos(phi / 2.0);
            double nz = bz / B, nxr = b1r / B, nxi = b1i / B;
            /* α = cos(φ/2) - i nz sin(φ/2);  β = -i (B1/B) sin(φ/2) */
            double ar = ch, ai = -(nz * sh);
            double br = nxi * sh, bi = -(nxr * sh);
            /* Mxy' = 2 conj(α) β Mz + conj(α)^2 Mxy - β^2 conj(Mxy) */
            double t1r, t1i, t2r, t2i, t3r, t3i, ca2r, ca2i, b2r, b2i;
            cmul(2.0 * ar, -(2.0 * ai), br, bi, &t1r, &t1i);
            t1r = t1r * zz;
            t1i = t1i * zz;
            cmul(ar, -ai, ar, -ai, &ca2r, &ca2i);
            cmul(ca2r, ca2i, xr, xi, &t2r, &t2i);
            cmul(br, bi, br, bi, &b2r, &b2i);
            cmul(b2r, b2i, xr, -xi, &t3r, &t3i);
            double nxr2 = (t1r + t2r) - t3r;
            double nxi2 = (t1i + t2i) - t3i;
            /* Mz' = (|α|^2 - |β|^2) Mz - 2 Re(α β conj(Mxy)) */
            double aa = hypot(ar, ai), bb = hypot(br, bi);
            double abr, abi, pr, pi_;
            cmul(ar, ai, br, bi, &abr, &abi);
            cmul(abr, abi, xr, -xi, &pr, &pi_);
            double nz2 = (aa * aa - bb * bb) * zz - 2.0 * pr;
            xr = nxr2;
            xi = nxi2;
            zz = nz2;
            /* relaxation */
            double e2 = exp(-q->dt[n] / p->T2[s]);
            xr = xr * e2;
            xi = xi * e2;
            double e1 = exp(-q->dt[n] / p->T1[s]);
            zz = zz * e1 + p->rho[s] * (1.0 - e1);
            if (q->adc[n + 1] && nadc > 0) {
                double sr, si;
                cmul(xr, xi, cos(q->psi[n + 1]), sin(q->psi[n + 1]), &sr, &si);
                for (int32_t c = 0; c < p->nc; ++c) {
                    const double *w = p->csm + 2 * (s + (int64_t)c * p->ns);
                    double vr, vi;
                    cmul(sr, si, w[0], w[1], &vr, &vi);
                    double *o = acc + 2 * (sample + (int64_t)c * nadc);
                    o[0] += vr;
                    o[1] += vi;
                }
                sample++;
            }
        }
        cmul(xr, xi, cos(q->psi[l]), sin(q->psi[l]), &xr, &xi);
        mxy[2 * s] = xr;
        mxy[2 * s + 1] = xi;
        mz[s] = zz;
    }
}

typedef struct or_part {
    const or_phantom *p;
    const or_sequence *q;
    uint32_t method;
    int32_t k;
    int64_t s0, s1, nadc;
    double *mxy, *mz, *acc;
} or_part;

static void *run_part(void *arg)
{
    or_part *w = (or_part *)arg;
    if (w->q->exc[w->k])
        excitation_block(w->p, w->q, w->method, w->k, w->s0, w->s1, w->mxy, w->mz, w->acc, w->nadc);
    else
        precession_block(w->p, w->q, w->method, w->k, w->s0, w->s1, w->mxy, w->mz, w->acc, w->nadc);
    return NULL;
}

/* run_sim_time_iter! (SimulatorCore.jl:96-152) restated: blocks in order,
 * spins split into `nthreads` contiguous parts (POSIX threads), each part
 * accumulating into its own slice, slices summed in part order after each
 * block (Simulate.jl:185 sums the thread dimension).
 * sig: (nadc_total x nc) column-major complex, overwritten.
 * mxy (complex) / mz: initial state in, final state out.
 * Returns 0 on success, -1 on bad arguments, -2 on allocation failure. */
int oracle_simulate(const or_phantom *p, const or_sequence *q, uint32_t method, double *mxy, double *mz,
                    double *sig, int64_t sig_rows, int nthreads)
{
    if (!p || !q || p->ns < 0 || p->nc < 1 || q->nt < 1) return -1;
    int64_t nadc_total = oracle_count_adc(q);
    if (sig_rows != nadc_total) return -1;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    memset(sig, 0, sizeof(double) * 2 * (size_t)nadc_total * (size_t)p->nc);
    int64_t max_adc = 0;
    for (int32_t k = 0; k < q->nblocks; ++k) {
        int64_t a = block_adc(q, k);
        if (a > max_adc) max_adc = a;
    }
    size_t slice = 2 * (size_t)(max_adc > 0 ? max_adc : 1) * (size_t)p->nc;
    double *acc = (double *)calloc(slice * (size_t)nthreads, sizeof(double));
    or_part *parts = (or_part *)calloc((size_t)nthreads, sizeof(or_part));
    pthread_t *tid = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    if (!acc || !parts || !tid) {
        free(acc);
        free(parts);
        free(tid);
        return -2;
    }
    int64_t sample0 = 0;
    for (int32_t k = 0; k < q->nblocks; ++k) {
        int64_t nadc = block_adc(q, k);
        memset(acc, 0, sizeof(double) * slice * (size_t)nthreads);
        for (int th = 0; th < nthreads; ++th) {
            or_part w = {p, q, method, k, p->ns * th / nthreads, p->ns * (th + 1) / nthreads, nadc, mxy, mz,
                         acc + slice * (size_t)th};
            parts[th] = w;
        }
        if (nthreads == 1) {
            run_part(&parts[0]);
        } else {
            int started = 0;
            for (int th = 0; th < nthreads; ++th) {
                if (pthread_create(&tid[th], NULL, run_part, &parts[th]) != 0) break;
                started++;
            }
            for (int th = 0; th < started; ++th) pthread_join(tid[th], NULL);
            for (int th = started; th < nthreads; ++th) run_part(&parts[th]);
        }
        for (int th = 0; th < nthreads; ++th) {
            const double *a = acc + slice * (size_t)th;
            for (int32_t c = 0; c < p->nc; ++c)
                for (int64_t j = 0; j < nadc; ++j) {
                    double *o = sig + 2 * (sample0 + j + (int64_t)c * nadc_total);
                    const double *v = a + 2 * (j + (int64_t)c * nadc);
                    o[0] += v[0];
                    o[1] += v[1];
                }
        }
        sample0 += nadc;
    }
    free(acc);
    free(parts);
    free(tid);
    return 0;
}

/* transpose(states)·csm (BlochHighOrderSimulatitonMethod.jl:17-20):
 * states (ns x nadc) column-major complex, csm (ns x nc), sig (nadc x nc). */
void oracle_coil_combine(int64_t ns, int64_t nadc, int32_t nc, const double *states, const double *csm,
                         double *sig)
{
    for (int32_t c = 0; c < nc; ++c)
        for (int64_t j = 0; j < nadc; ++j) {
            double sr = 0.0, si = 0.0;
            for (int64_t s = 0; s < ns; ++s) {
                double vr, vi;
                const double *a = states + 2 * (s + j * ns);
                const double *w = csm + 2 * (s + (int64_t)c * ns);
                cmul(a[0], a[1], w[0], w[1], &vr, &vi);
                sr += vr;
                si += vi;
            }
            sig[2 * (j + (int64_t)c * nadc)] = sr;
            sig[2 * (j + (int64_t)c * nadc) + 1] = si;
        }
}

int oracle_abi_version(void) { return 1; }
