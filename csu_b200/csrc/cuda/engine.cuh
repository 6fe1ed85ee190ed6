// engine.cuh -- device data structures and per-cell helpers of the residual-and-update engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "physics.cuh"
#include "ext80.cuh"
#include "lsqdd.cuh"
#include "viscous.cuh"
#include "sa.cuh"
#include "sacc.cuh"
#include "sst.cuh"

namespace csu {

constexpr int BLOCK = 256;
constexpr int MAX_SWEEPS = 64;

template <int MODEL>
struct Model {
    static constexpr int NV = MODEL == 0 ? 4 : (MODEL == 1 ? 5 : 6); // conserved variables
    static constexpr int NX = NV - 4;                                // transported scalars
    static constexpr int NP = NV + 1;                                // primitives r u v p T (nt | k w)
};

// Scalar settings, passed by value to every kernel.
struct Prm {
    Gas gas;
    int nc, nf, nb;
    int order, scheme, laminar, sa, sst, axi, turb1order, limiter_type, stages, dt_local_n, tube, n_linear;
    int lsq_exact;      // least squares: 0 precomputed FP64 weights (not bit-exact), 1 x87 model for every
                        // component, 2 certified double-double + x87 model for the rest (bit-exact)
    int visc;           // laminar, SA or SST: temperature gradient and viscous fluxes
    int visc_blazek;    // SA face gradients with the directional correction (saInterFaceB)
    int sa_cc;          // saCC: SA with the density-gradient terms (saCC.c)
    double lim_k, vol_max, e_fix, r_lim, p_out, t_wall, pr, pr_t, w_imp, cfl, sigma, mach_inf, sref;
    double pin[7];
    double pref20[6];   // limiterUpdate type 0 reference squares (limiter.c:49-59)
    double q_inf, p_inf;// solverCalcCoeff3 dynamic pressure and pressure (solver.c:1348-1352)
    double sst_b1, o_wall_factor;
    SstK sst_k;         // SST constants (sstInit)
    double tmax;        // tube end time
    double conv_tol;    // stop when res[0] <= conv_tol * res0[0], res0 the largest residual so far (0: never)
    int iter_cap;       // freeze the solve (done = 2) once its counter reaches this (0: never)
    int lim_func;       // limiter function: 0 Venkatakrishnan (limiterV2), 1 Barth-Jespersen (limiterBJ)
    int cell0;          // first cell of this solve (packs: cells [cell0, cell0 + nc), block aligned)
    int blk0, nblk;     // its cell blocks (residual-norm partial sums)
    int wall0, nwall;   // its wall faces in the wall-coefficient array
    int blk32;          // DPLUR blocks in FP32
    int sa_isrc;        // SA + DPLUR: the source's implicit part in the nt diagonal (dQ holds it per cell)
    int defer_fin;      // DPLUR: an iteration's k_finalize may run beside the next one's gradients and fluxes
    int mit_early;      // SA + DPLUR: k_face_mit writes the face eddy viscosity (from the primitives alone) for
                        // the blocks and the diagonal, which then need not wait for k_flux; k_flux skips it
    int implicit_local_dt;
    int cfl_ramp_iters; // CFL ramp (0: constant CFL)
    double cfl_max;
};

// Device scalars updated by the kernels themselves (one per solve).
struct Scalars {
    double dt;                            // global step of the running iteration
    double t;                             // physical time (tube)
    unsigned long long dtmin_bits;        // running min of local steps (non-negative double bits)
    unsigned long long sweep_max[MAX_SWEEPS]; // max |dx0| per DPLUR sweep (implicit.c:1023-1032)
    unsigned long long qmin_bits[6], qmax_bits[6]; // limiter type 1 global min/max (ordered bits)
    double res0[6];
    double res[6];
    double coef[4];
    int iter;                             // solverSolve loop counter of the next iteration
    int dt_local;                         // solver->dtLocal
    int status;                           // 0 or CSU_ERR_*
    int done;                             // converged / tube end reached
    int stop_after;                       // tube: this iteration reaches tmax
    int hist_row;                         // next history row
    int steps;                            // iterations completed in this call
    int have_res0;                        // res0 recorded
    int fresh;                            // state set from outside: the prologue derives W and the step
    int frozen;                           // (status | done) as the last DPLUR k_finalize found them on entry, or
                                          // as the call found them (k_call_begin): the halt test of the kernels
                                          // that run beside a deferred k_finalize (halted_behind)
    int hist_cap;                         // rows available at hist
    double* hist;                         // history rows of this solve (or null)
};

struct Mesh {
    int nc, nf, nb;
    const int* npts;
    const int* nint;
    const int* nslot;
    const int* nei;
    const double* wx;
    const double* wy;
    const double* ex;
    const double* ey;
    const double* ldx;              // least squares: neighbour centre minus centroid
    const double* ldy;
    const unsigned long long* lm;   // [4][nc] x87 significands of a, b, c, det
    const int* les;                 // [4][nc] exponent << 1 | sign
    const unsigned long long* lrv;  // reciprocal of det's significand
    const double2* lq;              // [4][nc] a, b, c and 1/det as exact (h, l) double-doubles
    const int* fslot;
    const int* fnb;                 // [4][nc] neighbour across interior face slot j, else -1
    const double* omega;
    const double* sxh;
    const double* syh;
    const double* wall_d;
    const double* dslat;
    const int2* fe;
    const double2* fn;
    const double* fds;
    const double2* r0;
    const double2* r1;
    const double2* fd;              // centroid of e1 minus centroid of e0
    const double* fL;               // |fd|
    const int* bown;
    const int* bflag;
    const int* bold;
    const double2* bn;
    const double* bds;
    const double2* bd;              // boundary edge midpoint minus owner centroid
    const double* bL;               // |bd|
    const double2* bun;             // unit normal of meshCalcDS2 (unscaled)
    const double* bds2;             // |dS| of meshCalcDS2 (axisymmetric: times the mean y)
    const int* color;               // cell colour (LU-SGS)
    const int* color_cells;         // cells grouped by colour
};

struct State {
    double4* U4;  double* Ux;                 // conserved state (after the write-back clamps)
    double4* W4;  double* WT;  double* Wx;    // primitives of the cells
    double4* G4x; double4* G4y; double4* PH4; // gradients and limiter (r u v p)
    double* GTx;  double* GTy;                // temperature gradient (solverGrad_T, viscous models)
    double4* FV;                              // viscous face fluxes (x, y momentum, energy, nt)
    double* MIT;                              // face eddy viscosity of interior faces (SA, SST)
    double* FV5;                              // SST: 5th viscous component (omega)
    double* Gxx;  double* Gxy;  double* PHx;  // same for the scalars, [k][cell]
    double4* F4;  double* Fx;                 // face fluxes * |dS|: nf interior then nb boundary
    double4* R4;  double* Rx;                 // residual
    double* dtl;                              // local steps (RK) or Omega / Lc (implicit)
    double* dpart;                            // implicit diagonal before Omega/dt
    double4* X4[2]; double* Xx[2];            // DPLUR increments (ping-pong)
    double* blocks;                           // DPLUR blocks [(slot*NV + row)*NV + col][cell]
    float* blocks32;                          // the same in FP32 (mixed-precision DPLUR)
    double* part;                             // per-block partial sums of R^2 [block][NV]
    double* bcoef;                            // per reference boundary face: cp dSx, cp dSy, fx/q, fy/q
    double* bcoef2;                           // DPLUR: the second buffer (iterations alternate, so that a deferred
                                              // k_finalize sums one while the next k_flux writes the other)
    Scalars* sc;                              // one per solve
    const int* bsolve;                        // packs: solve of each cell block (null: one solve)
    const int* csolve;                        // packs: solve of each cell (null: one solve)
    double* dbg_ghost;                        // optional: ghost primitives [bface][NP] (reference order)
    unsigned long long* lsq_x87;              // running count of gradient slots left to the integer x87 model
    double* dQ;                               // SST LU-SGS: source Jacobians [6][cell] (sst_source_jacobians)
    int2* gfix;                               // gradient variables left to k_grad_fix: (cell, var | mask << 8)
    unsigned* gfix_n;                         // entries in gfix (k_grad appends, k_grad_fix reads, the k_flux
                                              // that follows empties it)
};

// ---------------------------------------------------------------- small helpers

__device__ __forceinline__ unsigned long long dbits(double x)
{
    return (unsigned long long)__double_as_longlong(x);
}

__device__ __forceinline__ double bitsd(unsigned long long b)
{
    return __longlong_as_double((long long)b);
}

// order-preserving map of any double onto unsigned 64-bit (for atomic min/max of signed values)
__device__ __forceinline__ unsigned long long ordbits(double x)
{
    unsigned long long b = dbits(x);
    return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}

__device__ __forceinline__ double ordbits_inv(unsigned long long b)
{
    return bitsd((b & 0x8000000000000000ULL) ? (b & 0x7fffffffffffffffULL) : ~b);
}

template <int MODEL>
__device__ __forceinline__ void loadU(const State& s, int nc, int i, double* q)
{
    double4 t = s.U4[i];
    q[0] = t.x; q[1] = t.y; q[2] = t.z; q[3] = t.w;
#pragma unroll
    for (int k = 4; k < Model<MODEL>::NV; k++) q[k] = s.Ux[(size_t)(k - 4) * nc + i];
}

template <int MODEL>
__device__ __forceinline__ void storeU(const State& s, int nc, int i, const double* q)
{
    s.U4[i] = make_double4(q[0], q[1], q[2], q[3]);
#pragma unroll
    for (int k = 4; k < Model<MODEL>::NV; k++) s.Ux[(size_t)(k - 4) * nc + i] = q[k];
}

// primitives in the reference layout r u v p T (nt | k w)
template <int MODEL>
__device__ __forceinline__ void loadP(const State& s, int nc, int i, double* P)
{
    double4 t = s.W4[i];
    P[0] = t.x; P[1] = t.y; P[2] = t.z; P[3] = t.w;
    P[4] = s.WT[i];
#pragma unroll
    for (int k = 5; k < Model<MODEL>::NP; k++) P[k] = s.Wx[(size_t)(k - 5) * nc + i];
}

template <int MODEL>
__device__ __forceinline__ void storeP(const State& s, int nc, int i, const double* P)
{
    s.W4[i] = make_double4(P[0], P[1], P[2], P[3]);
    s.WT[i] = P[4];
#pragma unroll
    for (int k = 5; k < Model<MODEL>::NP; k++) s.Wx[(size_t)(k - 5) * nc + i] = P[k];
}

// CFL of iteration `it`: the reference's constant CFL, or the geometric ramp extension
__device__ __forceinline__ double cfl_at(const Prm& p, int it)
{
    if (p.cfl_ramp_iters <= 0) return p.cfl;
    double f = it >= p.cfl_ramp_iters ? 1.0 : (double)it / p.cfl_ramp_iters;
    return p.cfl * pow(p.cfl_max / p.cfl, f);
}

// primitive index of gradient/limiter slot kk (solver.c:461-468, 515-522)
__device__ __forceinline__ constexpr int slot2p(int kk)
{
    return kk > 3 ? kk + 1 : kk;
}

// solverCalcPrimitive for one cell (solver.c:1153-1213): clamps write back into U (omLim = 0)
template <int MODEL>
__device__ __forceinline__ void clamp_prim(const Prm& p, double* U, double* P)
{
    P[0] = U[0];
    P[0] = fmax(P[0], p.r_lim);
    U[0] = P[0];
    double k = 0;
    if constexpr (MODEL == 2) {
        k = U[4] / P[0];
        if (k < 1e-14) {
            k = 1e-14;
            U[4] = P[0] * k;
        }
        P[5] = k;
        double om = U[5] / P[0];
        if (om <= 0.0) {
            om = 0.0;
            U[5] = P[0] * om;
        }
        P[6] = om;
    }
    double u = U[1] / P[0];
    double v = U[2] / P[0];
    P[1] = u;
    P[2] = v;
    double e = U[3] / P[0] - 0.5 * (u * u + v * v) - k;
    e = fmax(e, 7.176325e+02);
    double T = e2T(p.gas, e);
    if (T < 1) {
        T = 1;
        e = T2e(p.gas, T);
        U[3] = (e + 0.5 * (u * u + v * v) + k) * P[0];
    }
    P[4] = T;
    P[3] = p.gas.R * P[4] * P[0];
    if constexpr (MODEL == 1) {
        P[5] = U[4] / P[0];
        P[5] = fmax(P[5], 0);
        U[4] = P[5] * P[0];
    }
}

// solverLocalTimeStep without the CFL factor (solver.c:895-923), from an unclamped state
template <int MODEL>
__device__ __forceinline__ double local_step(const Prm& p, const double* U, double sxh, double syh, double omega)
{
    double k = 0;
    if constexpr (MODEL == 2) k = U[4] / U[0];
    double E = U[3] / U[0];
    double u = U[1] / U[0];
    double v = U[2] / U[0];
    double aux = (E - (u * u + v * v) / 2 - k);
    double T = e2T(p.gas, aux);
    double c = T2c(p.gas, T);
    double Lx = (fabs(u) + c) * sxh;
    double Ly = (fabs(v) + c) * syh;
    return omega / (Lx + Ly);
}

// boundaryCalcPrimitive for one boundary element (boundary.c:514-693). E0 = owner primitives.
template <int MODEL>
__device__ __forceinline__ void ghost_state(const Prm& p, int flag, double dSx, double dSy, double dS,
                                            const double* E0, double dwall, double* G)
{
    double PL[4] = {E0[0], E0[1], E0[2], E0[3]};
    double Pb[4];
    if (flag == 0) {
        if (dS > 0) {
            rotation(PL, dSx, dSy, dS);
            PL[1] = 0.0;
            rotation(PL, dSx, -dSy, dS);
        } else {
            PL[2] = 0.0;
        }
        for (int k = 0; k < 4; k++) G[k] = PL[k];
        G[4] = G[3] / (G[0] * p.gas.R);
    } else if (flag == 1) {
        bcInlet(p.gas, p.pin, PL, Pb, dSx / dS, dSy / dS);
        for (int k = 0; k < 4; k++) G[k] = Pb[k];
        G[4] = G[3] / (G[0] * p.gas.R);
    } else if (flag == 2) {
        bcOutlet(p.gas, p.p_out, PL, Pb, dSx / dS, dSy / dS);
        for (int k = 0; k < 4; k++) G[k] = Pb[k];
        G[4] = G[3] / (G[0] * p.gas.R);
    } else {
        if (p.laminar == 1 || p.sa == 1) {
            if (flag == 4) {
                G[0] = PL[3] / (p.gas.R * p.t_wall);
                G[1] = 0.0;
                G[2] = 0.0;
                G[3] = PL[3];
                G[4] = p.t_wall;
            } else {
                G[0] = PL[0];
                G[1] = 0.0;
                G[2] = 0.0;
                G[3] = PL[3];
                G[4] = G[3] / (G[0] * p.gas.R);
            }
        } else {
            if (dS > 0) {
                bcWall(p.gas, PL, Pb, dSx / dS, dSy / dS);
                for (int k = 0; k < 4; k++) G[k] = Pb[k];
            } else {
                PL[2] = 0.0;
                for (int k = 0; k < 4; k++) G[k] = PL[k];
            }
            G[4] = G[3] / (G[0] * p.gas.R);
        }
    }
    if constexpr (MODEL == 1) {
        if (flag == 0 || flag == 2) G[5] = E0[5];
        else if (flag == 1) G[5] = p.pin[5];
        else G[5] = 0.0;
    }
    if constexpr (MODEL == 2) {
        if (flag == 0 || flag == 2) {
            G[5] = E0[5];
            G[6] = E0[6];
        } else if (flag == 1) {
            G[5] = p.pin[5];
            G[6] = p.pin[6];
        } else {
            double n = sutherland(G[4]) / G[0];
            double d = dwall;
            double owall = p.o_wall_factor * 6 * n / (p.sst_b1 * d * d);
            G[5] = 1e-14;
            G[6] = owall;
        }
    }
}

// boundaryCalc / _sa / _sst for one boundary element (boundary.c:143-443): flux in the global frame,
// not yet multiplied by |dS|. E0 = owner primitives (first order).
template <int MODEL>
__device__ __forceinline__ void boundary_flux(const Prm& p, int flag, double dSx, double dSy, double dS,
                                              const double* E0, double* f)
{
    constexpr int NV = Model<MODEL>::NV;
    double PL[NV], Q[NV], Pb[4];
#pragma unroll
    for (int k = 0; k < 4; k++) PL[k] = E0[k];
#pragma unroll
    for (int k = 4; k < NV; k++) PL[k] = E0[k + 1];
    if (flag == 0) {
        rotation(PL, dSx, dSy, dS);
        Q[0] = PL[0]; Q[1] = -PL[1]; Q[2] = PL[2]; Q[3] = PL[3];
#pragma unroll
        for (int k = 4; k < NV; k++) Q[k] = PL[k];
        riemann<MODEL>(p.scheme, p.gas, p.e_fix, p.mach_inf, PL, Q, f);
    } else if (flag == 1) {
        bcInlet(p.gas, p.pin, PL, Pb, dSx / dS, dSy / dS);
        rotation(PL, dSx, dSy, dS);
        rotation(Pb, dSx, dSy, dS);
        Q[0] = Pb[0]; Q[1] = Pb[1]; Q[2] = Pb[2]; Q[3] = Pb[3];
#pragma unroll
        for (int k = 4; k < NV; k++) Q[k] = p.pin[k + 1];
        riemann<MODEL>(p.scheme, p.gas, p.e_fix, p.mach_inf, PL, Q, f);
    } else if (flag == 2) {
        bcOutlet(p.gas, p.p_out, PL, Pb, dSx / dS, dSy / dS);
        rotation(PL, dSx, dSy, dS);
        rotation(Pb, dSx, dSy, dS);
        Q[0] = Pb[0]; Q[1] = Pb[1]; Q[2] = Pb[2]; Q[3] = Pb[3];
#pragma unroll
        for (int k = 4; k < NV; k++) Q[k] = PL[k];
        riemann<MODEL>(p.scheme, p.gas, p.e_fix, p.mach_inf, PL, Q, f);
    } else {
        if (MODEL == 0 && p.laminar != 1) {
            bcWall(p.gas, PL, Pb, dSx / dS, dSy / dS);
            rotation(Pb, dSx, dSy, dS);
            fluxFree(p.gas, Pb, f);
        } else {
            rotation(PL, dSx, dSy, dS);
            Q[0] = PL[0]; Q[1] = -PL[1]; Q[2] = -PL[2]; Q[3] = PL[3];
#pragma unroll
            for (int k = 4; k < NV; k++) Q[k] = PL[k];
            riemann<MODEL>(p.scheme, p.gas, p.e_fix, p.mach_inf, PL, Q, f);
        }
    }
    rotation(f, dSx, -dSy, dS);
}

// ---------------------------------------------------------------- block reductions

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_min(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide minimum / maximum, valid in thread 0; every thread of the block calls them. They let a kernel
// take one atomic per block on a solve's scalar instead of one per warp: atomics on one address serialise
// at the L2, and one per warp of a 160k-cell grid costs microseconds.
__device__ __forceinline__ double block_min(double v)
{
    __shared__ double sh[BLOCK / 32];
    v = warp_min(v);
    __syncthreads(); // an earlier call may still read sh
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < BLOCK / 32; w++) v = fmin(v, sh[w]);
    return v;
}

template <int NT = BLOCK>
__device__ __forceinline__ double block_max(double v)
{
    __shared__ double sh[NT / 32];
    v = warp_max(v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < NT / 32; w++) v = fmax(v, sh[w]);
    return v;
}

// Block-wide sums of N values per thread; result valid in thread 0. Deterministic order.
template <int N, int NT = BLOCK>
__device__ __forceinline__ void block_sum(double* v, double (*sh)[NT / 32])
{
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < N; k++) {
        double x = warp_sum(v[k]);
        if (lane == 0) sh[k][w] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < N; k++) {
            double acc = 0.0;
            for (int j = 0; j < NT / 32; j++) acc += sh[k][j];
            v[k] = acc;
        }
    }
}

} // namespace csu
