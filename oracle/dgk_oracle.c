/*
 * CPU FP64 restatement of the reference's OKL kernels for the partition-parallel tet-DG RHS.
 *
 * TEST INFRASTRUCTURE ONLY: this library is the oracle that the GPU path is checked against, and the
 * CPU baseline that bench.py times beside it.  The product library (dgkernel_b200/libdgk.so) never
 * links or calls it.
 *
 * OCCA Serial semantics are reproduced literally: an `@outer` loop over partitions becomes a plain
 * `for (part)` (an OpenMP `parallel for` when threads > 1, as OCCA's OpenMP mode does), `@inner`
 * becomes a plain loop over elements, and the MATMUL macros sum jj = 0..cols-1 sequentially.  Build
 * with -ffp-contract=off so no FMA changes the rounding.  Every partition-local pointer is
 * `X_global + X_offsets[part]` as the generated `X_PART(part)` macro does
 * (runner/builder/builder.go:281-310).
 *
 * Citations are relative to the DGKernel project root.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NFACES 4

/* MATMUL_<M> / MATMUL_ADD_<M> (runner/builder/builder.go:355-410).  M is column-major
 * (M[jj*rows+ii]), the device-matrix layout of builder.go:378 and the static layout
 * `const double M[cols][rows]` of builder.go:251-252. */
static void matmul_part(const double *M, int rows, int cols, const double *in, double *out, long K, int add)
{
    for (int ii = 0; ii < rows; ++ii) {
        for (long elem = 0; elem < K; ++elem) {
            double sum = 0.0;
            for (int jj = 0; jj < cols; ++jj)
                sum += M[(long)jj * rows + ii] * in[elem * cols + jj];
            if (add)
                out[elem * rows + ii] += sum;
            else
                out[elem * rows + ii] = sum;
        }
    }
}

static int set_threads(int threads)
{
#ifdef _OPENMP
    if (threads < 1) threads = 1;
    omp_set_num_threads(threads);
    return threads;
#else
    (void)threads;
    return 1;
#endif
}

/* Generic MATMUL over all partitions: OUT_PART(p) (+)= M x IN_PART(p). */
void ora_matmul(const double *M, int rows, int cols, int npart, const int64_t *K,
                const double *in, const int64_t *in_off, double *out, const int64_t *out_off, int add)
{
    for (int p = 0; p < npart; ++p)
        matmul_part(M, rows, cols, in + in_off[p], out + out_off[p], K[p], add);
}

/* `differentiate` (tetnudg/tet_nudg_mesh_physical_derivative_test.go:921-1078): Ur/Us/Ut by MATMUL,
 * then DuDx = Rx*Ur + Sx*Us + Tx*Ut etc.  All node arrays share the offsets `off`.  Ur/Us/Ut are
 * caller-provided temporaries sized like U. */
void ora_differentiate(int Np, const double *Dr, const double *Ds, const double *Dt, int npart, const int64_t *K,
                       const int64_t *off, const double *U, const double *Rx, const double *Ry, const double *Rz,
                       const double *Sx, const double *Sy, const double *Sz, const double *Tx, const double *Ty,
                       const double *Tz, double *Ur, double *Us, double *Ut, double *DuDx, double *DuDy,
                       double *DuDz, int threads)
{
    set_threads(threads);
#pragma omp parallel for schedule(static) if (threads > 1)
    for (int part = 0; part < npart; ++part) {
        const long o = off[part];
        matmul_part(Dr, Np, Np, U + o, Ur + o, K[part], 0);
        matmul_part(Ds, Np, Np, U + o, Us + o, K[part], 0);
        matmul_part(Dt, Np, Np, U + o, Ut + o, K[part], 0);
        for (long k = 0; k < K[part]; ++k) {
            for (int n = 0; n < Np; ++n) {
                const long i = o + n + k * Np;
                DuDx[i] = Rx[i] * Ur[i] + Sx[i] * Us[i] + Tx[i] * Ut[i];
                DuDy[i] = Ry[i] * Ur[i] + Sy[i] * Us[i] + Ty[i] * Ut[i];
                DuDz[i] = Rz[i] * Ur[i] + Sz[i] * Us[i] + Tz[i] * Ut[i];
            }
        }
    }
}

/* Volume-only `computeRHS` (examples/3d_scalar_burgers_equation.go:295-346):
 * rhsu = -u * (ux + uy + uz). */
void ora_compute_rhs_volume(int Np, const double *Dr, const double *Ds, const double *Dt, int npart,
                            const int64_t *K, const int64_t *off, const double *u, const double *Rx,
                            const double *Ry, const double *Rz, const double *Sx, const double *Sy,
                            const double *Sz, const double *Tx, const double *Ty, const double *Tz, double *ur,
                            double *us, double *ut, double *rhsu, int threads)
{
    set_threads(threads);
#pragma omp parallel for schedule(static) if (threads > 1)
    for (int part = 0; part < npart; ++part) {
        const long o = off[part];
        matmul_part(Dr, Np, Np, u + o, ur + o, K[part], 0);
        matmul_part(Ds, Np, Np, u + o, us + o, K[part], 0);
        matmul_part(Dt, Np, Np, u + o, ut + o, K[part], 0);
        for (long elem = 0; elem < K[part]; ++elem) {
            for (int i = 0; i < Np; ++i) {
                const long idx = o + elem * Np + i;
                double ux = Rx[idx] * ur[idx] + Sx[idx] * us[idx] + Tx[idx] * ut[idx];
                double uy = Ry[idx] * ur[idx] + Sy[idx] * us[idx] + Ty[idx] * ut[idx];
                double uz = Rz[idx] * ur[idx] + Sz[idx] * us[idx] + Tz[idx] * ut[idx];
                rhsu[idx] = -u[idx] * (ux + uy + uz);
            }
        }
    }
}

/* `updateSolution` exactly as the reference writes it (examples/3d_scalar_burgers_equation.go:359-378):
 * resu = rka*resu + rkb*rhsu; u = u + resu. */
void ora_update_ref(int Np, int npart, const int64_t *K, const int64_t *off, double *u, double *resu,
                    const double *rhsu, double rka, double rkb)
{
    for (int part = 0; part < npart; ++part) {
        const long o = off[part];
        for (long elem = 0; elem < K[part]; ++elem)
            for (int i = 0; i < Np; ++i) {
                const long idx = o + elem * Np + i;
                resu[idx] = rka * resu[idx] + rkb * rhsu[idx];
                u[idx] = u[idx] + resu[idx];
            }
    }
}

/* Face exchange pick -> exchange -> place into per-partition P buffers
 * (utils/face_connector.go:143-187; runtime form of utils/face_connector_test.go:98-157).
 * pick lists are CSR over pairs (src*npart + dst); place lists CSR over (dst*npart + src).
 * `pbuf` is partition-local at face offsets `foff`. */
void ora_exchange(int npart, const double *u, const int64_t *uoff, const int64_t *pick_ptr,
                  const int64_t *pick_idx, const int64_t *place_ptr, const int64_t *place_idx, double *pbuf,
                  const int64_t *foff)
{
    for (int src = 0; src < npart; ++src)
        for (int dst = 0; dst < npart; ++dst) {
            const int64_t *pk = pick_idx + pick_ptr[src * npart + dst];
            const int64_t *pl = place_idx + place_ptr[dst * npart + src];
            const long n = (long)(pick_ptr[src * npart + dst + 1] - pick_ptr[src * npart + dst]);
            for (long i = 0; i < n; ++i)
                pbuf[foff[dst] + pl[i]] = u[uoff[src] + pk[i]];
        }
}

/* Strong-form Lax-Friedrichs surface term for f(u) = (u^2/2)(1,1,1):
 *   n.f = (u^2/2)(nx+ny+nz), lambda = |u| |nx+ny+nz|,
 *   du  = n.f(uM) - [ (n.f(uM)+n.f(uP))/2 + max(lamM,lamP)/2 (uM-uP) ],
 * returned times Fscale (the build's fixed form of documentation/DGKernel/example_application.md:300-334). */
static inline double lf_surface(double uM, double uP, double nsum, double fscale)
{
    const double fM = 0.5 * uM * uM * nsum;
    const double fP = 0.5 * uP * uP * nsum;
    const double lamM = fabs(uM) * fabs(nsum);
    const double lamP = fabs(uP) * fabs(nsum);
    const double C = lamM > lamP ? lamM : lamP;
    const double du = fM - (0.5 * (fM + fP) + 0.5 * C * (uM - uP));
    return fscale * du;
}

/* Full strong-form RHS, one partition (volume of examples/3d_scalar_burgers_equation.go:295-346 plus the
 * LF surface term lifted by MATMUL_LIFT):
 *   rhs = -u (ux+uy+uz) + LIFT (Fscale .* du)               (conservative = 0, the reference form)
 *   rhs = -(d/dx+d/dy+d/dz)(u^2/2) + LIFT (Fscale .* du)    (conservative = 1)
 * Arrays are partition-local; uP holds the P-buffer values at each face point; fmask is (4, Nfp). */
static void rhs_lf_part(int Np, int Nfp, const double *Dr, const double *Ds, const double *Dt, const double *LIFT,
                        const int32_t *fmask, long K, const double *u, const double *Rx, const double *Ry,
                        const double *Rz, const double *Sx, const double *Sy, const double *Sz, const double *Tx,
                        const double *Ty, const double *Tz, const double *nx, const double *ny, const double *nz,
                        const double *Fscale, const double *uP, double *rhs, double *ur, double *us, double *ut,
                        double *flux, double *w, int conservative)
{
    const int NF = NFACES * Nfp;
    const double *src = u;
    if (conservative) {
        for (long i = 0; i < K * Np; ++i) w[i] = 0.5 * u[i] * u[i];
        src = w;
    }
    matmul_part(Dr, Np, Np, src, ur, K, 0);
    matmul_part(Ds, Np, Np, src, us, K, 0);
    matmul_part(Dt, Np, Np, src, ut, K, 0);
    for (long elem = 0; elem < K; ++elem) {
        for (int i = 0; i < Np; ++i) {
            const long idx = elem * Np + i;
            double ux = Rx[idx] * ur[idx] + Sx[idx] * us[idx] + Tx[idx] * ut[idx];
            double uy = Ry[idx] * ur[idx] + Sy[idx] * us[idx] + Ty[idx] * ut[idx];
            double uz = Rz[idx] * ur[idx] + Sz[idx] * us[idx] + Tz[idx] * ut[idx];
            rhs[idx] = conservative ? -(ux + uy + uz) : -u[idx] * (ux + uy + uz);
        }
        for (int f = 0; f < NFACES; ++f)
            for (int i = 0; i < Nfp; ++i) {
                const long fid = elem * NF + f * Nfp + i;
                const double uM = u[elem * Np + fmask[f * Nfp + i]];
                flux[fid] = lf_surface(uM, uP[fid], nx[fid] + ny[fid] + nz[fid], Fscale[fid]);
            }
    }
    matmul_part(LIFT, Np, NF, flux, rhs, K, 1);
}

/* Standard Carpenter-Kennedy LSERK4 stage: resu = a*resu + dt*rhs; u = u + b*resu. */
static void lserk_part(long n, double *u, double *resu, const double *rhs, double a, double b, double dt)
{
    for (long i = 0; i < n; ++i) {
        resu[i] = a * resu[i] + dt * rhs[i];
        u[i] = u[i] + b * resu[i];
    }
}

/* One RHS evaluation over all partitions (exchange, then per-partition RHS); `rhs` is node-offset. */
void ora_rhs_lf(int Np, int Nfp, const double *Dr, const double *Ds, const double *Dt, const double *LIFT,
                const int32_t *fmask, int npart, const int64_t *K, const int64_t *noff, const int64_t *foff,
                const double *u, const double *Rx, const double *Ry, const double *Rz, const double *Sx,
                const double *Sy, const double *Sz, const double *Tx, const double *Ty, const double *Tz,
                const double *nx, const double *ny, const double *nz, const double *Fscale,
                const int64_t *pick_ptr, const int64_t *pick_idx, const int64_t *place_ptr,
                const int64_t *place_idx, double *pbuf, double *rhs, int conservative, int threads)
{
    const int NF = NFACES * Nfp;
    ora_exchange(npart, u, noff, pick_ptr, pick_idx, place_ptr, place_idx, pbuf, foff);
    set_threads(threads);
#pragma omp parallel for schedule(static) if (threads > 1)
    for (int p = 0; p < npart; ++p) {
        const long n = K[p] * Np;
        double *scratch = (double *)malloc(sizeof(double) * (size_t)(4 * n + K[p] * NF));
        const long o = noff[p], fo = foff[p];
        rhs_lf_part(Np, Nfp, Dr, Ds, Dt, LIFT, fmask, K[p], u + o, Rx + o, Ry + o, Rz + o, Sx + o, Sy + o, Sz + o,
                    Tx + o, Ty + o, Tz + o, nx + fo, ny + fo, nz + fo, Fscale + fo, pbuf + fo, rhs + o, scratch,
                    scratch + n, scratch + 2 * n, scratch + 4 * n, scratch + 3 * n, conservative);
        free(scratch);
    }
}

/* LSERK4 coefficients, Carpenter & Kennedy (examples/3d_scalar_burgers_equation.go:138-151). */
static const double RK4A[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                               -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
static const double RK4B[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                               1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                               2277821191437.0 / 14882151754819.0};

void ora_lserk_coefficients(double *a, double *b)
{
    memcpy(a, RK4A, sizeof(RK4A));
    memcpy(b, RK4B, sizeof(RK4B));
}

/* Time loop: nsteps x 5 LSERK4 stages of (exchange, RHS, update).  `stage0` selects the first stage
 * index and `nstages` the number of stages to run (nstages = 5*nsteps for whole steps).  u and resu are
 * node-offset arrays, updated in place.  Returns the number of stages executed. */
long ora_run(int Np, int Nfp, const double *Dr, const double *Ds, const double *Dt, const double *LIFT,
             const int32_t *fmask, int npart, const int64_t *K, const int64_t *noff, const int64_t *foff,
             double *u, double *resu, const double *Rx, const double *Ry, const double *Rz, const double *Sx,
             const double *Sy, const double *Sz, const double *Tx, const double *Ty, const double *Tz,
             const double *nx, const double *ny, const double *nz, const double *Fscale, const int64_t *pick_ptr,
             const int64_t *pick_idx, const int64_t *place_ptr, const int64_t *place_idx, double dt, int stage0,
             long nstages, int conservative, int threads)
{
    long nnode = noff[npart], nface = foff[npart];
    double *pbuf = (double *)calloc((size_t)nface, sizeof(double));
    double *rhs = (double *)calloc((size_t)nnode, sizeof(double));
    for (long s = 0; s < nstages; ++s) {
        const int st = (int)((stage0 + s) % 5);
        ora_rhs_lf(Np, Nfp, Dr, Ds, Dt, LIFT, fmask, npart, K, noff, foff, u, Rx, Ry, Rz, Sx, Sy, Sz, Tx, Ty, Tz,
                   nx, ny, nz, Fscale, pick_ptr, pick_idx, place_ptr, place_idx, pbuf, rhs, conservative, threads);
        set_threads(threads);
#pragma omp parallel for schedule(static) if (threads > 1)
        for (int p = 0; p < npart; ++p)
            lserk_part(K[p] * Np, u + noff[p], resu + noff[p], rhs + noff[p], RK4A[st], RK4B[st], dt);
    }
    free(pbuf);
    free(rhs);
    return nstages;
}

int ora_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_num_procs();
#else
    return 1;
#endif
}

/* ---- artificial viscosity with a modal shock sensor (the build's fixed formulas; parity unpinned) ----
 *
 * Sensor (Persson & Peraire): uhat = Vinv u per element (orthonormal modes, element/library/gonudg/
 * simplex3dp.go:15-36, order i, j, k of vandermonde3d.go:15-42); S = log10(sum over modes of total degree N
 * of uhat^2 / sum over all modes of uhat^2); activation sigma = 0 for S < s0 - kappa, 1 for S > s0 + kappa,
 * else (1 + sin(pi (S - s0) / (2 kappa))) / 2.  Viscosity eps_e = eps0 sigma_e h_e / N with h_e = 2 / max
 * of the element's Fscale.  Learned mode (2): sigma = MLP(uhat / |uhat|) (nin -> 32 -> 32 -> 1, tanh, tanh,
 * sigmoid) where the MLP output lies outside (conf_lo, conf_hi), the PP sigma inside that band; mode 3 is the
 * same with outputs at or below conf_lo read as a smooth element, sigma = 0.
 *
 * Viscous term (BR1, central fluxes): q_d = D_d u + LIFT (Fscale n_d (uP - uM) / 2), d = x, y, z; then
 * rhs += eps_e sum_d D_d q_d + LIFT (Fscale 1/2 sum_d n_d (epsP qP_d - epsM qM_d)). */

static double pp_sigma(double S, double s0, double kappa)
{
    if (!(S >= s0 - kappa)) return 0.0; /* also S = -inf (an element with no energy) */
    if (S > s0 + kappa) return 1.0;
    return 0.5 * (1.0 + sin(M_PI * (S - s0) / (2.0 * kappa)));
}

double ora_mlp_forward1(int nin, const double *p, const double *x)
{
    const double *W1 = p, *b1 = W1 + 32 * nin, *W2 = b1 + 32, *b2 = W2 + 32 * 32, *w3 = b2 + 32, *b3 = w3 + 32;
    double h1[32], h2[32];
    for (int o = 0; o < 32; ++o) {
        double s = b1[o];
        for (int i = 0; i < nin; ++i) s += W1[o * nin + i] * x[i];
        h1[o] = tanh(s);
    }
    for (int o = 0; o < 32; ++o) {
        double s = b2[o];
        for (int i = 0; i < 32; ++i) s += W2[o * 32 + i] * h1[i];
        h2[o] = tanh(s);
    }
    double z = b3[0];
    for (int i = 0; i < 32; ++i) z += w3[i] * h2[i];
    return 1.0 / (1.0 + exp(-z));
}

static void modal_features(int Np, const double *Vinv, const int32_t *top, const double *ue, double *uh,
                           double *S, double *feat)
{
    double tot = 0.0, hi = 0.0;
    for (int i = 0; i < Np; ++i) {
        double s = 0.0;
        for (int j = 0; j < Np; ++j) s += Vinv[(long)j * Np + i] * ue[j];
        uh[i] = s;
        tot += s * s;
        if (top[i]) hi += s * s;
    }
    *S = tot > 0.0 ? log10(hi / tot) : -INFINITY;
    if (feat) {
        const double inv = tot > 0.0 ? 1.0 / sqrt(tot) : 0.0;
        for (int i = 0; i < Np; ++i) feat[i] = uh[i] * inv;
    }
}

void ora_sensor(int Np, const double *Vinv, const int32_t *top, long K, const double *u, double s0, double kappa,
                double *S, double *sigma, double *feat)
{
    double uh[256];
    for (long e = 0; e < K; ++e) {
        modal_features(Np, Vinv, top, u + e * Np, uh, &S[e], feat ? feat + e * Np : NULL);
        sigma[e] = pp_sigma(S[e], s0, kappa);
    }
}

void ora_rhs_av(int Np, int Nfp, int N, const double *Dr, const double *Ds, const double *Dt, const double *LIFT,
                const double *Vinv, const int32_t *top, const int32_t *fmask, long K, const double *u,
                const double *Rx, const double *Ry, const double *Rz, const double *Sx, const double *Sy,
                const double *Sz, const double *Tx, const double *Ty, const double *Tz, const double *nx,
                const double *ny, const double *nz, const double *Fscale, const int64_t *vmapP, int mode, double eps0,
                double s0, double kappa, const double *mlp, double conf_lo, double conf_hi, double *rhs,
                double *eps_out, int threads)
{
    const int NF = NFACES * Nfp;
    const double *geo[9] = {Rx, Ry, Rz, Sx, Sy, Sz, Tx, Ty, Tz};
    const double *nrm[3] = {nx, ny, nz};
    double *eps = (double *)malloc(sizeof(double) * (size_t)K);
    double *q = (double *)malloc(sizeof(double) * (size_t)(3 * K * Np));
    set_threads(threads);
    /* pass 1: sensor, eps, q */
#pragma omp parallel for schedule(static) if (threads > 1)
    for (long e = 0; e < K; ++e) {
        double uh[256], ft[256], ur[256], us[256], ut[256], fl[3][512];
        const double *ue = u + e * Np;
        double S, sig = 0.0;
        modal_features(Np, Vinv, top, ue, uh, &S, ft);
        if (mode == 1) {
            sig = pp_sigma(S, s0, kappa);
        } else if (mode == 2 || mode == 3) {
            sig = ora_mlp_forward1(Np, mlp, ft);
            if (sig > conf_lo && sig < conf_hi) sig = pp_sigma(S, s0, kappa);
            else if (mode == 3 && sig <= conf_lo) sig = 0.0;
        }
        double fmax = 0.0;
        for (int m = 0; m < NF; ++m) fmax = fmax > Fscale[e * NF + m] ? fmax : Fscale[e * NF + m];
        eps[e] = eps0 * sig * (2.0 / fmax) / N;
        for (int i = 0; i < Np; ++i) {
            double a = 0.0, b = 0.0, c = 0.0;
            for (int j = 0; j < Np; ++j) {
                a += Dr[(long)j * Np + i] * ue[j];
                b += Ds[(long)j * Np + i] * ue[j];
                c += Dt[(long)j * Np + i] * ue[j];
            }
            ur[i] = a, us[i] = b, ut[i] = c;
        }
        for (int m = 0; m < NF; ++m) {
            const long fid = e * NF + m;
            const double jump = 0.5 * (u[vmapP[fid]] - ue[fmask[m]]) * Fscale[fid];
            for (int d = 0; d < 3; ++d) fl[d][m] = nrm[d][fid] * jump;
        }
        for (int d = 0; d < 3; ++d)
            for (int i = 0; i < Np; ++i) {
                const long idx = e * Np + i;
                double s = geo[d][idx] * ur[i] + geo[3 + d][idx] * us[i] + geo[6 + d][idx] * ut[i];
                for (int m = 0; m < NF; ++m) s += LIFT[(long)m * Np + i] * fl[d][m];
                q[(long)d * K * Np + idx] = s;
            }
    }
    /* pass 2: LF RHS plus the viscous divergence */
#pragma omp parallel for schedule(static) if (threads > 1)
    for (long e = 0; e < K; ++e) {
        double ur[256], us[256], ut[256], flux[512];
        const double *ue = u + e * Np;
        for (int i = 0; i < Np; ++i) {
            double a = 0.0, b = 0.0, c = 0.0;
            for (int j = 0; j < Np; ++j) {
                a += Dr[(long)j * Np + i] * ue[j];
                b += Ds[(long)j * Np + i] * ue[j];
                c += Dt[(long)j * Np + i] * ue[j];
            }
            ur[i] = a, us[i] = b, ut[i] = c;
        }
        for (int i = 0; i < Np; ++i) {
            const long idx = e * Np + i;
            const double ux = Rx[idx] * ur[i] + Sx[idx] * us[i] + Tx[idx] * ut[i];
            const double uy = Ry[idx] * ur[i] + Sy[idx] * us[i] + Ty[idx] * ut[i];
            const double uz = Rz[idx] * ur[i] + Sz[idx] * us[i] + Tz[idx] * ut[i];
            rhs[idx] = -ue[i] * (ux + uy + uz);
        }
        /* eps * sum_d D_d q_d */
        for (int d = 0; d < 3; ++d) {
            const double *qd = q + (long)d * K * Np + e * Np;
            for (int i = 0; i < Np; ++i) {
                double a = 0.0, b = 0.0, c = 0.0;
                for (int j = 0; j < Np; ++j) {
                    a += Dr[(long)j * Np + i] * qd[j];
                    b += Ds[(long)j * Np + i] * qd[j];
                    c += Dt[(long)j * Np + i] * qd[j];
                }
                const long idx = e * Np + i;
                rhs[idx] += eps[e] * (geo[d][idx] * a + geo[3 + d][idx] * b + geo[6 + d][idx] * c);
            }
        }
        for (int m = 0; m < NF; ++m) {
            const long fid = e * NF + m;
            const long gP = vmapP[fid], gM = e * Np + fmask[m];
            const double ePs = eps[gP / Np];
            double vis = 0.0;
            for (int d = 0; d < 3; ++d)
                vis += nrm[d][fid] * (ePs * q[(long)d * K * Np + gP] - eps[e] * q[(long)d * K * Np + gM]);
            flux[m] = lf_surface(u[gM], u[gP], nx[fid] + ny[fid] + nz[fid], Fscale[fid]) + 0.5 * Fscale[fid] * vis;
        }
        for (int i = 0; i < Np; ++i) {
            double s = 0.0;
            for (int m = 0; m < NF; ++m) s += LIFT[(long)m * Np + i] * flux[m];
            rhs[e * Np + i] += s;
        }
    }
    if (eps_out) memcpy(eps_out, eps, sizeof(double) * (size_t)K);
    free(eps);
    free(q);
}

long ora_run_av(int Np, int Nfp, int N, const double *Dr, const double *Ds, const double *Dt, const double *LIFT,
                const double *Vinv, const int32_t *top, const int32_t *fmask, long K, double *u, double *resu,
                const double *Rx, const double *Ry, const double *Rz, const double *Sx, const double *Sy,
                const double *Sz, const double *Tx, const double *Ty, const double *Tz, const double *nx,
                const double *ny, const double *nz, const double *Fscale, const int64_t *vmapP, int mode, double eps0,
                double s0, double kappa, const double *mlp, double conf_lo, double conf_hi, double dt, int stage0,
                long nstages, int threads)
{
    double *rhs = (double *)calloc((size_t)(K * Np), sizeof(double));
    for (long s = 0; s < nstages; ++s) {
        const int st = (int)((stage0 + s) % 5);
        ora_rhs_av(Np, Nfp, N, Dr, Ds, Dt, LIFT, Vinv, top, fmask, K, u, Rx, Ry, Rz, Sx, Sy, Sz, Tx, Ty, Tz, nx, ny,
                   nz, Fscale, vmapP, mode, eps0, s0, kappa, mlp, conf_lo, conf_hi, rhs, NULL, threads);
        lserk_part(K * Np, u, resu, rhs, RK4A[st], RK4B[st], dt);
    }
    free(rhs);
    return nstages;
}
