// kernels.cuh -- the residual-and-update kernels.
//
// One residual evaluation (solverCalcR, solver.c:685) is three passes over HBM:
//   k_grad   per cell:  gathers neighbour primitives (ghost states of boundary neighbours are evaluated on
//                       the fly from the cell's own state: a ghost is only ever its owner's neighbour),
//                       least-squares gradient + Venkatakrishnan limiter          (solver.c:451-548)
//   k_flux   per face:  MUSCL states, rotation, Riemann flux * |dS| for interior faces, first-order
//                       boundary fluxes for boundary faces; one launch, block-uniform split (inter 550-644,
//                       boundary.c:143-443)
//   k_rk / k_impl per cell: gathers the signed face fluxes in the reference's order (inter 646-667, then
//                       boundary faces, then the axisymmetric source) and fuses the state update that follows
//                       (solverRK, or the implicit diagonal and DPLUR blocks), the next stage's primitives
//                       with their clamps, local time steps and residual-norm partial sums.
// Nothing is scattered, so no atomics are needed on the state; the only atomics are order-free min/max of
// scalars. Kernels exit immediately once the solve's device status says "done" or "error", so whole
// iteration sequences can be captured in one CUDA graph.
#pragma once
#include "engine.cuh"

namespace csu {

__device__ __forceinline__ bool halted(const Scalars* sc)
{
    return (sc->status | sc->done) != 0;
}

// The halt test of the kernels that, in DPLUR, may run beside the previous iteration's k_finalize (limiter
// bounds, gradients, face fluxes): the flags k_finalize is writing are not read; `frozen` (the flags one
// k_finalize behind) is. A solve halted by iteration i's k_finalize therefore still gets iteration i + 1's
// gradients and face fluxes, of the state it stopped at, and nothing after them: its later iterations
// either skip these kernels or recompute the same values, whichever flag value they read.
__device__ __forceinline__ bool halted_behind(const Prm& p, const Scalars* sc)
{
    return p.defer_fin ? sc->frozen != 0 : halted(sc);
}

// Solve of a cell block (in a pack every block holds cells of one solve) and of a cell; cells of the
// solve are [p.cell0, p.cell0 + p.nc), the rest of its last block is padding.
__device__ __forceinline__ int block_solve(const State& s)
{
    return s.bsolve ? s.bsolve[blockIdx.x] : 0;
}

__device__ __forceinline__ int cell_solve(const State& s, int c)
{
    return s.csolve ? s.csolve[c] : 0;
}

__device__ __forceinline__ bool cell_in(const Prm& p, int c)
{
    return (unsigned)(c - p.cell0) < (unsigned)p.nc;
}

// ------------------------------------------------------------------------------------------------
// k_prim: W = primitives of clamp(U), U := clamp(U) (solverCalcPrimitive cell loop). With dt: the local
// step of the unclamped state first (solverCalcDt precedes solverCalcR, solver.c:1868-1869).
// ------------------------------------------------------------------------------------------------
template <int MODEL>
__global__ void __launch_bounds__(BLOCK) k_prim(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                const __grid_constant__ State s, int with_dt, int only_fresh)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    const int sid = block_solve(s);
    const Prm& p = P[sid];
    Scalars* const sc = s.sc + sid;
    // prologue of a pack: solves carried over from another pack keep their primitives and step
    if (only_fresh && !sc->fresh) return;
    int c = blockIdx.x * BLOCK + threadIdx.x;
    double lmin = __longlong_as_double(0x7ff0000000000000LL);
    if (cell_in(p, c)) {
        double U[NV], P[NP];
        loadU<MODEL>(s, m.nc, c, U);
        if (with_dt) {
            double l = local_step<MODEL>(p, U, m.sxh[c], m.syh[c], m.omega[c]);
            s.dtl[c] = cfl_at(p, sc->iter) * l;
            lmin = l;
        }
        clamp_prim<MODEL>(p, U, P);
        storeU<MODEL>(s, m.nc, c, U);
        storeP<MODEL>(s, m.nc, c, P);
    }
    if (with_dt) {
        double v = block_min(lmin);
        if (threadIdx.x == 0 && !(v > bitsd(0x7fefffffffffffffULL))) atomicMin(&sc->dtmin_bits, dbits(v));
    }
}

// ------------------------------------------------------------------------------------------------
// k_grad: solverUpdateGrad + the limiter loop of inter (solver.c:451-548).
// DBG also records ghost primitives (boundaryCalcPrimitive) in reference order.
// LSQ selects the least-squares arithmetic (Prm::lsq_exact): 0 precomputed FP64 weights, 1 the integer x87
// model (ext80.cuh) for every component, 2 the FP64 x87 emulation and certified double-double solve of
// lsqdd.cuh, with the integer model only for the rare components those cannot decide (k_grad_fix).
// ------------------------------------------------------------------------------------------------

// x87 constants a, b, c, det of cell c (solver.c:1063-1073, evaluated on the host in long double)
__device__ __forceinline__ void lsq_consts(const Mesh& m, int nc, int c, X80* K)
{
#pragma unroll
    for (int q = 0; q < 4; q++) {
        int es = m.les[(size_t)q * nc + c];
        K[q].m = m.lm[(size_t)q * nc + c];
        K[q].e = es >> 1;
        K[q].s = es & 1;
    }
}

// limiterCalc epsilon^2 of slot kk (limiter.c:98-119); aux = (K sqrt(omega / omega_max))^3 for type 0
__device__ __forceinline__ double limiter_eps2(const Prm& p, const Scalars* sc, int kk, double aux)
{
    if (p.limiter_type == 0) return p.pref20[kk] * aux;
    // type 1 (limiter.c:61-94): ((max - min) K)^2 over the solve's cells, from k_minmax
    double a2 = (ordbits_inv(sc->qmax_bits[kk]) - ordbits_inv(sc->qmin_bits[kk])) * p.lim_k;
    return a2 * a2;
}

// One gradient component pair of cell c for primitive vi (T: 4) with the integer x87 model, gathering the
// neighbours again; also the cell's value of the primitive and its range over the cell and the neighbours
// (the limiter's inputs). Only the rare components the FP64 path cannot decide come here (k_grad_fix).
template <int MODEL>
__device__ __forceinline__ double2 lsq_slot_x87(const Prm& p, const Mesh& m, const State& s, int c, int vi,
                                                double* u0p, double* qminp, double* qmaxp)
{
    constexpr int NP = Model<MODEL>::NP;
    const int nc = m.nc;
    double P0[NP];
    loadP<MODEL>(s, nc, c, P0);
    double u0 = 0.0;
#pragma unroll
    for (int k = 0; k < NP; k++)
        if (k == vi) u0 = P0[k];
    *u0p = u0;
    *qminp = u0;
    *qmaxp = u0;
    X80 XA = x80_zero(0), XB = x80_zero(0);
    const int np = m.npts[c];
    const double dw = m.wall_d ? m.wall_d[c] : 0.0;
    for (int j = 0; j < np; j++) {
        int n = m.nei[(size_t)j * nc + c];
        double Pn[NP];
        if (n < nc) {
            loadP<MODEL>(s, nc, n, Pn);
        } else {
            int b = n - nc;
            double2 dSv = m.bn[b];
            ghost_state<MODEL>(p, m.bflag[b], dSv.x, dSv.y, m.bds[b], P0, dw, Pn);
        }
        double un = 0.0;
#pragma unroll
        for (int k = 0; k < NP; k++)
            if (k == vi) un = Pn[k];
        double du = un - u0;
        *qmaxp = fmax(*qmaxp, un);
        *qminp = fmin(*qminp, un);
        XA = x80_add(XA, x80_from_double(m.ldx[(size_t)j * nc + c] * du));
        XB = x80_add(XB, x80_from_double(m.ldy[(size_t)j * nc + c] * du));
    }
    X80 K[4];
    lsq_consts(m, nc, c, K);
    unsigned long long rv = m.lrv[c];
    X80 nx = x80_add(x80_mul(K[2], XA), x80_neg(x80_mul(K[1], XB)));
    X80 ny = x80_add(x80_mul(x80_neg(K[1]), XA), x80_mul(K[0], XB));
    atomicAdd(s.lsq_x87, 1ULL);
    return make_double2(x80_to_double(x80_div_pre(nx, K[3], rv)), x80_to_double(x80_div_pre(ny, K[3], rv)));
}

// ------------------------------------------------------------------------------------------------
// k_minmax: limiterUpdate type 1 (limiter.c:61-94): the minimum and maximum over the solve's cells of each
// limited primitive (slot 4 reads P[5], limiter.c:66-70), as order-preserving bits (exact, order-free).
// k_minmax_init resets them, one block per solve.
// ------------------------------------------------------------------------------------------------
__global__ void k_minmax_init(State s)
{
    Scalars* sc = s.sc + blockIdx.x;
    if (threadIdx.x < 6) {
        sc->qmin_bits[threadIdx.x] = ~0ULL;
        sc->qmax_bits[threadIdx.x] = 0ULL;
    }
}

template <int MODEL>
__global__ void __launch_bounds__(BLOCK) k_minmax(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                  const __grid_constant__ State s)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    const int sid = block_solve(s);
    const Prm& p = P[sid];
    Scalars* const sc = s.sc + sid;
    if (halted_behind(p, sc)) return;
    const int c = blockIdx.x * BLOCK + threadIdx.x;
    const bool ok = cell_in(p, c);
    double W[NP];
    if (ok) loadP<MODEL>(s, m.nc, c, W);
#pragma unroll
    for (int kk = 0; kk < NV; kk++) {
        double v = ok ? W[kk == 4 ? 5 : kk] : 0.0;
        const bool use = ok && !isnan(v); // fmin / fmax skip NaN operands (limiter.c:84-85)
        unsigned long long lo = use ? ordbits(v) : ~0ULL, hi = use ? ordbits(v) : 0ULL;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&sc->qmin_bits[kk], lo);
            atomicMax(&sc->qmax_bits[kk], hi);
        }
    }
}

template <int MODEL, bool DBG, int LSQ>
__global__ void __launch_bounds__(BLOCK, MODEL == 0 ? 3 : 2) k_grad(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                const __grid_constant__ State s)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    const int sid = block_solve(s);
    const Prm& p = P[sid];
    Scalars* const sc = s.sc + sid;
    const int c = blockIdx.x * BLOCK + threadIdx.x;
    if (!cell_in(p, c) || halted_behind(p, sc)) return;
    {
        const int nc = m.nc;
        double P0[NP];
        loadP<MODEL>(s, nc, c, P0);
        double gx[NV], gy[NV], qmin[NV], qmax[NV];
        X80 XA[NV], XB[NV], TA = x80_zero(0), TB = x80_zero(0);
        DD AX[NV], AY[NV], TX = {0.0, 0.0}, TY = {0.0, 0.0};
        bool sum_ok = true;
        double gtx = 0.0, gty = 0.0;
        const bool visc = p.visc != 0;
#pragma unroll
        for (int kk = 0; kk < NV; kk++) {
            gx[kk] = 0.0;
            gy[kk] = 0.0;
            qmin[kk] = P0[slot2p(kk)];
            qmax[kk] = P0[slot2p(kk)];
            if (LSQ == 1) {
                XA[kk] = x80_zero(0);
                XB[kk] = x80_zero(0);
            }
            if (LSQ == 2) {
                AX[kk].h = AX[kk].l = 0.0;
                AY[kk].h = AY[kk].l = 0.0;
            }
        }
        const int np = m.npts[c];
        const double dw = m.wall_d ? m.wall_d[c] : 0.0;
        // the FP64 path runs the neighbour loop rolled: one copy of the gather, ghost state and x87 steps
        constexpr int JU = LSQ == 2 ? 1 : 4;
#pragma unroll JU
        for (int j = 0; j < 4; j++) {
            if (j < np) {
                int n = m.nei[(size_t)j * nc + c];
                double Pn[NP];
                if (n < nc) {
                    loadP<MODEL>(s, nc, n, Pn);
                } else {
                    int b = n - nc;
                    double2 dSv = m.bn[b];
                    ghost_state<MODEL>(p, m.bflag[b], dSv.x, dSv.y, m.bds[b], P0, dw, Pn);
                    if (DBG) {
                        int bo = m.bold[b];
                        for (int k = 0; k < NP; k++) s.dbg_ghost[(size_t)bo * NP + k] = Pn[k];
                    }
                }
                if (LSQ != 0) {
                    // solverCalcGrad3 (solver.c:1063-1070): double products summed in long double
                    double dxj = m.ldx[(size_t)j * nc + c], dyj = m.ldy[(size_t)j * nc + c];
                    if (visc) {
                        double dT = Pn[4] - P0[4];
                        if (LSQ == 1) {
                            TA = x80_add(TA, x80_from_double(dxj * dT));
                            TB = x80_add(TB, x80_from_double(dyj * dT));
                        } else if (j == 0) {
                            TX.h = dxj * dT;
                            TY.h = dyj * dT;
                        } else if (j == 1) {
                            TX = x87_sum2(TX.h, dxj * dT, sum_ok);
                            TY = x87_sum2(TY.h, dyj * dT, sum_ok);
                        } else {
                            TX = x87_sum_add(TX, dxj * dT, sum_ok);
                            TY = x87_sum_add(TY, dyj * dT, sum_ok);
                        }
                    }
#pragma unroll
                    for (int kk = 0; kk < NV; kk++) {
                        double du = Pn[slot2p(kk)] - P0[slot2p(kk)];
                        if (LSQ == 1) {
                            XA[kk] = x80_add(XA[kk], x80_from_double(dxj * du));
                            XB[kk] = x80_add(XB[kk], x80_from_double(dyj * du));
                        } else if (j == 0) {
                            AX[kk].h = dxj * du;
                            AY[kk].h = dyj * du;
                        } else if (j == 1) {
                            AX[kk] = x87_sum2(AX[kk].h, dxj * du, sum_ok);
                            AY[kk] = x87_sum2(AY[kk].h, dyj * du, sum_ok);
                        } else {
                            AX[kk] = x87_sum_add(AX[kk], dxj * du, sum_ok);
                            AY[kk] = x87_sum_add(AY[kk], dyj * du, sum_ok);
                        }
                        qmax[kk] = fmax(qmax[kk], Pn[slot2p(kk)]);
                        qmin[kk] = fmin(qmin[kk], Pn[slot2p(kk)]);
                    }
                } else {
                    double wxj = m.wx[(size_t)j * nc + c], wyj = m.wy[(size_t)j * nc + c];
                    if (visc) {
                        double dT = Pn[4] - P0[4];
                        gtx += wxj * dT;
                        gty += wyj * dT;
                    }
#pragma unroll
                    for (int kk = 0; kk < NV; kk++) {
                        double du = Pn[slot2p(kk)] - P0[slot2p(kk)];
                        gx[kk] += wxj * du;
                        gy[kk] += wyj * du;
                        qmax[kk] = fmax(qmax[kk], Pn[slot2p(kk)]);
                        qmin[kk] = fmin(qmin[kk], Pn[slot2p(kk)]);
                    }
                }
            }
        }
        if (LSQ != 0) {
            // dUx = (c A - b B) / (a c - b b), dUy = (-b A + a B) / (a c - b b) in long double (solver.c:1072-1073)
            if (LSQ == 1) {
                X80 K[4];
                lsq_consts(m, nc, c, K);
                unsigned long long rv = m.lrv[c];
#pragma unroll
                for (int kk = 0; kk < NV; kk++) {
                    X80 nx = x80_add(x80_mul(K[2], XA[kk]), x80_neg(x80_mul(K[1], XB[kk])));
                    X80 ny = x80_add(x80_mul(x80_neg(K[1]), XA[kk]), x80_mul(K[0], XB[kk]));
                    gx[kk] = x80_to_double(x80_div_pre(nx, K[3], rv));
                    gy[kk] = x80_to_double(x80_div_pre(ny, K[3], rv));
                }
                if (visc) {
                    // solverGrad_T (solver.c:477-490): the same least squares on T
                    X80 nx = x80_add(x80_mul(K[2], TA), x80_neg(x80_mul(K[1], TB)));
                    X80 ny = x80_add(x80_mul(x80_neg(K[1]), TA), x80_mul(K[0], TB));
                    gtx = x80_to_double(x80_div_pre(nx, K[3], rv));
                    gty = x80_to_double(x80_div_pre(ny, K[3], rv));
                }
            } else {
                // a, b, c and 1/det as double-doubles, precomputed on the host
                double2 qa = m.lq[c], qb = m.lq[(size_t)nc + c], qc = m.lq[(size_t)2 * nc + c];
                double2 qr = m.lq[(size_t)3 * nc + c];
                DD ka = {qa.x, qa.y}, kb = {qb.x, qb.y}, kc = {qc.x, qc.y}, R = {qr.x, qr.y};
                // bit 2 kk + (0: x, 1: y) set where the cheap certified solve cannot decide; slot NV is T
                unsigned need = 0;
#pragma unroll
                for (int kk = 0; kk < NV; kk++) {
                    if (!lsq_certified(kc, kb, R, AX[kk], AY[kk], &gx[kk])) need |= 1u << (2 * kk);
                    if (!lsq_certified(ka, kb, R, AY[kk], AX[kk], &gy[kk])) need |= 2u << (2 * kk);
                }
                if (visc) {
                    if (!lsq_certified(kc, kb, R, TX, TY, &gtx)) need |= 1u << (2 * NV);
                    if (!lsq_certified(ka, kb, R, TY, TX, &gty)) need |= 2u << (2 * NV);
                }
                if (!sum_ok) need = visc ? (4u << (2 * NV)) - 1u : (1u << (2 * NV)) - 1u;
                // one out-of-loop copy of the exact-numerator solve; what that cannot decide (about one
                // component in a thousand) is left to k_grad_fix and the integer x87 model, whose registers
                // and code would otherwise slow every cell of this kernel
                unsigned xneed = 0;
#pragma unroll 1
                while (need) {
                    const int b = __ffs(need) - 1;
                    need &= need - 1;
                    const int kk = b >> 1, comp = b & 1;
                    DD X = TX, Y = TY;
#pragma unroll
                    for (int q = 0; q < NV; q++) {
                        if (q == kk) {
                            X = AX[q];
                            Y = AY[q];
                        }
                    }
                    double g = 0.0;
                    bool ok = sum_ok && (comp ? lsq_exact_numerator(ka, kb, R, Y, X, &g)
                                              : lsq_exact_numerator(kc, kb, R, X, Y, &g));
                    if (!ok) xneed |= 1u << b;
                    if (kk == NV) {
                        if (comp) gty = g;
                        else gtx = g;
                    }
#pragma unroll
                    for (int q = 0; q < NV; q++) {
                        if (q == kk) {
                            if (comp) gy[q] = g;
                            else gx[q] = g;
                        }
                    }
                }
                // one k_grad_fix entry per (cell, variable) with undecided components
#pragma unroll 1
                for (int q = 0; q <= NV; q++) {
                    const unsigned mk = (xneed >> (2 * q)) & 3u;
                    if (mk) s.gfix[atomicAdd(s.gfix_n, 1u)] = make_int2(c, q | (int)(mk << 8));
                }
            }
        }
        if (visc) {
            s.GTx[c] = gtx;
            s.GTy[c] = gty;
        }
        double phi[NV];
#pragma unroll
        for (int kk = 0; kk < NV; kk++) phi[kk] = 1.0;
        if (p.order == 2) {
            // limiterCalc (limiter.c:98-119), type 0: eps^2 = q_inf^2 (K sqrt(omega/omega_max))^3
            double aux = p.lim_k * sqrt(m.omega[c] / p.vol_max);
            aux = aux * aux * aux;
            double ee[NV];
#pragma unroll
            for (int kk = 0; kk < NV; kk++) ee[kk] = limiter_eps2(p, sc, kk, aux);
#pragma unroll JU
            for (int j = 0; j < 4; j++) {
                if (j < np) {
                    double exj = m.ex[(size_t)j * nc + c], eyj = m.ey[(size_t)j * nc + c];
#pragma unroll
                    for (int kk = 0; kk < NV; kk++) {
                        double d2 = (gx[kk] * exj + gy[kk] * eyj);
                        double phi0 = p.lim_func == 1 ? limiterBJ(P0[slot2p(kk)], qmin[kk], qmax[kk], d2)
                                                      : limiterV2(P0[slot2p(kk)], qmin[kk], qmax[kk], d2, ee[kk]);
                        phi[kk] = j == 0 ? phi0 : fmin(phi[kk], phi0);
                    }
                }
            }
        }
        s.G4x[c] = make_double4(gx[0], gx[1], gx[2], gx[3]);
        s.G4y[c] = make_double4(gy[0], gy[1], gy[2], gy[3]);
        s.PH4[c] = make_double4(phi[0], phi[1], phi[2], phi[3]);
#pragma unroll
        for (int kk = 4; kk < NV; kk++) {
            s.Gxx[(size_t)(kk - 4) * nc + c] = gx[kk];
            s.Gxy[(size_t)(kk - 4) * nc + c] = gy[kk];
            s.PHx[(size_t)(kk - 4) * nc + c] = phi[kk];
        }
    }
}

// ------------------------------------------------------------------------------------------------
// k_grad_fix: the gradient components neither k_grad's certified solve nor its exact x87 numerator could
// decide, entry (cell, variable kk (NV: temperature), mask of x / y): both components of the variable with
// the integer x87 model (lsq_slot_x87), the undecided ones taken from it, then the variable's limiter
// (limiterCalc) from the final gradient, as k_grad computes it. Grid-stride over the entries; k_flux, which
// always follows, empties the list for the next gradient launch.
// ------------------------------------------------------------------------------------------------
template <int MODEL>
__global__ void __launch_bounds__(BLOCK) k_grad_fix(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                    const __grid_constant__ State s)
{
    constexpr int NV = Model<MODEL>::NV;
    const unsigned n = *s.gfix_n;
    const int nc = m.nc;
    for (unsigned e = blockIdx.x * BLOCK + threadIdx.x; e < n; e += gridDim.x * BLOCK) {
        const int2 w = s.gfix[e];
        const int c = w.x, kk = w.y & 0xff, mask = w.y >> 8;
        const int sid = cell_solve(s, c);
        const Prm& p = P[sid];
        const Scalars* sc = s.sc + sid;
        double u0, qmin, qmax;
        const double2 gg = lsq_slot_x87<MODEL>(p, m, s, c, kk < NV ? slot2p(kk) : 4, &u0, &qmin, &qmax);
        // the components k_grad decided are already in place
        double* gxp = kk == NV ? s.GTx + c : kk < 4 ? reinterpret_cast<double*>(s.G4x + c) + kk
                                                      : s.Gxx + (size_t)(kk - 4) * nc + c;
        double* gyp = kk == NV ? s.GTy + c : kk < 4 ? reinterpret_cast<double*>(s.G4y + c) + kk
                                                      : s.Gxy + (size_t)(kk - 4) * nc + c;
        const double gx = (mask & 1) ? gg.x : *gxp, gy = (mask & 2) ? gg.y : *gyp;
        *gxp = gx;
        *gyp = gy;
        if (kk < NV && p.order == 2) {
            double aux = p.lim_k * sqrt(m.omega[c] / p.vol_max);
            aux = aux * aux * aux;
            const double ee = limiter_eps2(p, sc, kk, aux);
            const int np = m.npts[c];
            double phi = 1.0;
#pragma unroll 1
            for (int j = 0; j < np; j++) {
                double exj = m.ex[(size_t)j * nc + c], eyj = m.ey[(size_t)j * nc + c];
                double d2 = (gx * exj + gy * eyj);
                double phi0 = p.lim_func == 1 ? limiterBJ(u0, qmin, qmax, d2) : limiterV2(u0, qmin, qmax, d2, ee);
                phi = j == 0 ? phi0 : fmin(phi, phi0);
            }
            if (kk < 4) reinterpret_cast<double*>(s.PH4 + c)[kk] = phi;
            else s.PHx[(size_t)(kk - 4) * nc + c] = phi;
        }
    }
}

// The owner's gradients a boundary face's viscous flux uses: u, v, T, then nt (SA) or k (SST), then the rho
// gradient (SA: saCC's density terms) or omega (SST).
template <int MODEL>
__device__ __forceinline__ void owner_visc_gradients(const State& s, int nc, int c, double* gvx, double* gvy)
{
    double4 a = s.G4x[c], bb = s.G4y[c];
    gvx[0] = a.y; gvx[1] = a.z; gvx[2] = s.GTx[c];
    gvy[0] = bb.y; gvy[1] = bb.z; gvy[2] = s.GTy[c];
    gvx[3] = MODEL >= 1 ? s.Gxx[c] : 0.0;
    gvy[3] = MODEL >= 1 ? s.Gxy[c] : 0.0;
    gvx[4] = MODEL == 2 ? s.Gxx[(size_t)nc + c] : (MODEL == 1 ? a.x : 0.0);
    gvy[4] = MODEL == 2 ? s.Gxy[(size_t)nc + c] : (MODEL == 1 ? bb.x : 0.0);
}

// Viscous flux of boundary face b (device order; fi its slot in the face arrays) from its owner c's
// primitives E0 and gradients: boundaryFaceViscFlux (laminar.c:128-346), saBoundaryFaceViscFlux (sa.c:370-692)
// or its saCC variant, sstBoundaryFaceViscFlux (sst.c:202-547); stored in FV (and FV5) at fi.
template <int MODEL>
__device__ __forceinline__ void bface_visc(const Prm& p, const Mesh& m, const State& s, int b, int fi, int c,
                                           int flag, double dSx, double dSy, const double* E0, const double* gvx,
                                           const double* gvy, double2 bdv, double bLv)
{
    if constexpr (MODEL == 2) {
        double2 un = m.bun[b];
        double fv[5];
        sst_boundary_flux(p.gas, p.sst_k, p.pr, p.pr_t, p.t_wall, p.pin, flag, gvx, gvy, E0, m.wall_d[c], dSx, dSy,
                          bdv.x, bdv.y, bLv, un.x, un.y, m.bds2[b], fv);
        s.FV[fi] = make_double4(fv[0], fv[1], fv[2], fv[3]);
        s.FV5[fi] = fv[4];
    } else if constexpr (MODEL == 1) {
        double2 un = m.bun[b];
        double fv[4];
        if (p.sa_cc)
            sacc_boundary_flux(p.gas, p.pr, p.pr_t, p.t_wall, p.pin, flag, gvx, gvy, E0, dSx, dSy, bdv.x, bdv.y,
                               bLv, un.x, un.y, m.bds2[b], fv);
        else
            sa_boundary_flux(p.gas, p.pr, p.pr_t, p.t_wall, p.pin, flag, gvx, gvy, E0, dSx, dSy, bdv.x, bdv.y, bLv,
                             un.x, un.y, m.bds2[b], fv);
        s.FV[fi] = make_double4(fv[0], fv[1], fv[2], fv[3]);
    } else {
        if (p.laminar == 1) {
            double2 un = m.bun[b];
            double fv[3];
            laminar_boundary(p.gas, p.pr, p.t_wall, p.pin, flag, gvx, gvy, E0, dSx, dSy, bdv.x, bdv.y, bLv, un.x,
                             un.y, m.bds2[b], fv);
            s.FV[fi] = make_double4(fv[0], fv[1], fv[2], 0.0);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// k_wall_data: what the reference's surface writers read after its last iteration (solverWriteSolution2
// recomputes the cell and ghost primitives of the final state, solver.c:2038, while the gradients stay
// those of the last residual evaluation): per boundary face, the ghost primitives of the current cell
// primitives (into dbg_ghost, reference order) and the boundary viscous flux of the current primitives and
// gradients (into FV).
// ------------------------------------------------------------------------------------------------
template <int MODEL>
__global__ void __launch_bounds__(BLOCK) k_wall_data(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                     const __grid_constant__ State s)
{
    constexpr int NP = Model<MODEL>::NP;
    const int b = blockIdx.x * BLOCK + threadIdx.x;
    if (b >= m.nb) return;
    const int nc = m.nc, c = m.bown[b];
    const Prm& p = P[cell_solve(s, c)];
    const int flag = m.bflag[b];
    const double2 dSv = m.bn[b];
    const double dSx = dSv.x, dSy = dSv.y, dS = m.bds[b];
    double E0[NP], G[NP];
    loadP<MODEL>(s, nc, c, E0);
    ghost_state<MODEL>(p, flag, dSx, dSy, dS, E0, m.wall_d ? m.wall_d[c] : 0.0, G);
    const int bo = m.bold[b];
#pragma unroll
    for (int k = 0; k < NP; k++) s.dbg_ghost[(size_t)bo * NP + k] = G[k];
    if (p.visc) {
        double gvx[5], gvy[5];
        owner_visc_gradients<MODEL>(s, nc, c, gvx, gvy);
        bface_visc<MODEL>(p, m, s, b, m.nf + b, c, flag, dSx, dSy, E0, gvx, gvy, m.bd[b], m.bL[b]);
    }
}

// One interior face of k_flux (inter, solver.c:550-644, and the viscous face terms): MUSCL reconstruction,
// rotation, Riemann flux times |dS|, and the face's viscous flux and eddy viscosity. The two cells'
// primitives r u v p T, gradients and limiters of r u v p come in as values (read from global memory, or
// from a shared-memory window of cells); everything else is read here.
template <int MODEL>
__device__ __forceinline__ void interior_face(const Prm& p, const Mesh& m, const State& s, int f, int2 e,
                                              double4 w0, double t0, double4 gx0, double4 gy0, double4 ph0,
                                              double4 w1, double t1, double4 gx1, double4 gy1, double4 ph1)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    const int nc = m.nc;
    double2 dSv = m.fn[f];
    double dSx = dSv.x, dSy = dSv.y, dS = m.fds[f];
    double PL[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double PR[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double A[NP], B[NP];
    A[0] = w0.x; A[1] = w0.y; A[2] = w0.z; A[3] = w0.w; A[4] = t0;
    B[0] = w1.x; B[1] = w1.y; B[2] = w1.z; B[3] = w1.w; B[4] = t1;
#pragma unroll
    for (int k = 5; k < NP; k++) {
        A[k] = s.Wx[(size_t)(k - 5) * nc + e.x];
        B[k] = s.Wx[(size_t)(k - 5) * nc + e.y];
    }
    if (p.order == 2) {
        double2 r0 = m.r0[f], r1 = m.r1[f];
        double g0x[4] = {gx0.x, gx0.y, gx0.z, gx0.w}, g0y[4] = {gy0.x, gy0.y, gy0.z, gy0.w};
        double g1x[4] = {gx1.x, gx1.y, gx1.z, gx1.w}, g1y[4] = {gy1.x, gy1.y, gy1.z, gy1.w};
        double f0[4] = {ph0.x, ph0.y, ph0.z, ph0.w}, f1[4] = {ph1.x, ph1.y, ph1.z, ph1.w};
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            PL[kk] = A[kk] + (g0x[kk] * r0.x + g0y[kk] * r0.y) * f0[kk];
            PR[kk] = B[kk] + (g1x[kk] * r1.x + g1y[kk] * r1.y) * f1[kk];
        }
#pragma unroll
        for (int kk = 4; kk < NV; kk++) {
            if (p.turb1order) {
                PL[kk] = A[kk + 1];
                PR[kk] = B[kk + 1];
            } else {
                size_t o = (size_t)(kk - 4) * nc;
                PL[kk] = A[kk + 1] + (s.Gxx[o + e.x] * r0.x + s.Gxy[o + e.x] * r0.y) * s.PHx[o + e.x];
                PR[kk] = B[kk + 1] + (s.Gxx[o + e.y] * r1.x + s.Gxy[o + e.y] * r1.y) * s.PHx[o + e.y];
            }
        }
    } else {
#pragma unroll
        for (int kk = 0; kk < NV; kk++) {
            PL[kk] = A[slot2p(kk)];
            PR[kk] = B[slot2p(kk)];
        }
    }
    if constexpr (MODEL == 2) {
        const double4 a = gx0, b = gy0, cc = gx1, d = gy1;
        double g0x[5] = {a.y, a.z, s.GTx[e.x], s.Gxx[e.x], s.Gxx[(size_t)nc + e.x]};
        double g0y[5] = {b.y, b.z, s.GTy[e.x], s.Gxy[e.x], s.Gxy[(size_t)nc + e.x]};
        double g1x[5] = {cc.y, cc.z, s.GTx[e.y], s.Gxx[e.y], s.Gxx[(size_t)nc + e.y]};
        double g1y[5] = {d.y, d.z, s.GTy[e.y], s.Gxy[e.y], s.Gxy[(size_t)nc + e.y]};
        double2 dd = m.fd[f];
        double fv[5], mit;
        sst_face_flux(p.gas, p.sst_k, p.pr, p.pr_t, g0x, g0y, g1x, g1y, A, B, m.wall_d[e.x], m.wall_d[e.y], dd.x,
                      dd.y, m.fL[f], dSx, dSy, fv, &mit);
        s.FV[f] = make_double4(fv[0], fv[1], fv[2], fv[3]);
        s.FV5[f] = fv[4];
        s.MIT[f] = mit;
    } else if constexpr (MODEL == 1) {
        const double4 a = gx0, b = gy0, cc = gx1, d = gy1;
        double g0x[5] = {a.y, a.z, s.GTx[e.x], s.Gxx[e.x], a.x}, g0y[5] = {b.y, b.z, s.GTy[e.x], s.Gxy[e.x], b.x};
        double g1x[5] = {cc.y, cc.z, s.GTx[e.y], s.Gxx[e.y], cc.x}, g1y[5] = {d.y, d.z, s.GTy[e.y], s.Gxy[e.y], d.x};
        double2 dd = m.fd[f];
        double fv[4], mit;
        if (p.sa_cc)
            sacc_face_flux(p.gas, p.pr, p.pr_t, g0x, g0y, g1x, g1y, A, B, dSx, dSy, fv, &mit);
        else
            sa_face_flux(p.gas, p.pr, p.pr_t, p.visc_blazek, g0x, g0y, g1x, g1y, A, B, dd.x, dd.y, m.fL[f], dSx,
                         dSy, fv, &mit);
        s.FV[f] = make_double4(fv[0], fv[1], fv[2], fv[3]);
        if (!p.mit_early) s.MIT[f] = mit;
    } else if (p.laminar == 1) {
        const double4 a = gx0, b = gy0, cc = gx1, d = gy1;
        double g0x[3] = {a.y, a.z, s.GTx[e.x]}, g0y[3] = {b.y, b.z, s.GTy[e.x]};
        double g1x[3] = {cc.y, cc.z, s.GTx[e.y]}, g1y[3] = {d.y, d.z, s.GTy[e.y]};
        double2 dd = m.fd[f];
        double fv[3];
        laminar_face(p.gas, p.pr, g0x, g0y, g1x, g1y, A, B, dd.x, dd.y, m.fL[f], dSx, dSy, fv);
        s.FV[f] = make_double4(fv[0], fv[1], fv[2], 0.0);
    }
    rotation(PL, dSx, dSy, dS);
    rotation(PR, dSx, dSy, dS);
    double fl[NV];
    riemann<MODEL>(p.scheme, p.gas, p.e_fix, p.mach_inf, PL, PR, fl);
    rotation(fl, dSx, -dSy, dS);
    s.F4[f] = make_double4(fl[0] * dS, fl[1] * dS, fl[2] * dS, fl[3] * dS);
#pragma unroll
    for (int kk = 4; kk < NV; kk++) s.Fx[(size_t)(kk - 4) * (m.nf + m.nb) + f] = fl[kk] * dS;
}

// One boundary face b of k_flux (device order): the boundary flux of boundary.c:143-464 from the owner's
// first-order state and the ghost, the face's viscous flux, and the wall pressure and friction terms of
// solverCalcCoeff3 when `coef`.
template <int MODEL>
__device__ __forceinline__ void boundary_face(const Prm* __restrict__ P, const Mesh& m, const State& s, int b,
                                              const int* wall_rank, int coef)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    const int nc = m.nc;
    int c = m.bown[b];
    const int sid = cell_solve(s, c);
    const Prm& p = P[sid];
    if (halted_behind(p, s.sc + sid)) return;
    int flag = m.bflag[b];
    double2 dSv = m.bn[b];
    double dSx = dSv.x, dSy = dSv.y, dS = m.bds[b];
    double E0[NP];
    loadP<MODEL>(s, nc, c, E0);
    double fl[NV];
    boundary_flux<MODEL>(p, flag, dSx, dSy, dS, E0, fl);
    int fi = m.nf + b;
    double sc = dS > 0 ? dS : 0.0;
    s.F4[fi] = dS > 0 ? make_double4(fl[0] * dS, fl[1] * dS, fl[2] * dS, fl[3] * dS)
                      : make_double4(0.0, 0.0, 0.0, 0.0);
#pragma unroll
    for (int kk = 4; kk < NV; kk++) s.Fx[(size_t)(kk - 4) * (m.nf + m.nb) + fi] = dS > 0 ? fl[kk] * sc : 0.0;
    double gvx[5], gvy[5];
    double2 bdv = make_double2(0.0, 0.0);
    double bLv = 0.0;
    if (p.visc) {
        owner_visc_gradients<MODEL>(s, nc, c, gvx, gvy);
        bdv = m.bd[b];
        bLv = m.bL[b];
        bface_visc<MODEL>(p, m, s, b, fi, c, flag, dSx, dSy, E0, gvx, gvy, bdv, bLv);
    }
    if (coef && (flag == 3 || flag == 4)) {
        double* const bc = coef == 2 ? s.bcoef2 : s.bcoef;
        double G[NP];
        ghost_state<MODEL>(p, flag, dSx, dSy, dS, E0, m.wall_d ? m.wall_d[c] : 0.0, G);
        double cp = (G[3] - p.p_inf) / p.q_inf;
        int r = wall_rank[b];
        bc[(size_t)r * 4 + 0] = cp * dSx;
        bc[(size_t)r * 4 + 1] = cp * dSy;
        double fx = 0.0, fy = 0.0;
        if (p.visc) friction_wall(gvx, gvy, E0, dSx, dSy, bdv.x, bdv.y, bLv, &fx, &fy);
        bc[(size_t)r * 4 + 2] = p.visc ? fx / p.q_inf : 0.0;
        bc[(size_t)r * 4 + 3] = p.visc ? fy / p.q_inf : 0.0;
    }
}

// ------------------------------------------------------------------------------------------------
// k_flux: interior faces (blocks [0, nbi)) and boundary faces (blocks [nbi, ...)).
// coef: also record the wall pressure-coefficient terms of solverCalcCoeff3 (solver.c:1360-1385).
// ------------------------------------------------------------------------------------------------
template <int MODEL, int FB>
__global__ void __launch_bounds__(FB) k_flux(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                             const __grid_constant__ State s, int nbi, const int* wall_rank,
                                             int coef)
{
    // k_grad_fix (always launched just before) has read its list: empty it for the next gradient launch
    if (blockIdx.x == 0 && threadIdx.x == 0 && s.gfix_n) *s.gfix_n = 0;
    if ((int)blockIdx.x < nbi) {
        int f = blockIdx.x * FB + threadIdx.x;
        if (f >= m.nf) return;
        int2 e = m.fe[f];
        const int sid = cell_solve(s, e.x);
        const Prm& p = P[sid];
        if (halted_behind(p, s.sc + sid)) return;
        const double4 z4 = make_double4(0.0, 0.0, 0.0, 0.0);
        const bool grad = p.order == 2 || p.visc;
        interior_face<MODEL>(p, m, s, f, e, s.W4[e.x], s.WT[e.x], grad ? s.G4x[e.x] : z4, grad ? s.G4y[e.x] : z4,
                             p.order == 2 ? s.PH4[e.x] : z4, s.W4[e.y], s.WT[e.y], grad ? s.G4x[e.y] : z4,
                             grad ? s.G4y[e.y] : z4, p.order == 2 ? s.PH4[e.y] : z4);
    } else {
        int b = (blockIdx.x - nbi) * FB + threadIdx.x;
        if (b >= m.nb) return;
        boundary_face<MODEL>(P, m, s, b, wall_rank, coef);
    }
}

// ------------------------------------------------------------------------------------------------
// k_flux_st: k_flux with the interior faces' cell data staged in shared memory. Faces are sorted by their
// lower cell, so a block of FB faces starts at its first face's lower cell and most of its cells, both
// sides, lie in the next WIN cells (94 % of the faces on the 160,000-cell ramp for FB 128, WIN 256). The
// block loads that window's primitives r u v p T (and, when the faces need them, gradients and limiters of
// r u v p) with coalesced loads, then each face reads its cells from the window, or from global memory when
// a cell lies outside it. Same arithmetic, same bits as k_flux; the boundary faces are k_flux's.
// ------------------------------------------------------------------------------------------------
template <int MODEL, int FB, int WIN>
__global__ void __launch_bounds__(FB) k_flux_st(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                const __grid_constant__ State s, int nbi, const int* wall_rank,
                                                int coef)
{
    // k_grad_fix (always launched just before) has read its list: empty it for the next gradient launch
    if (blockIdx.x == 0 && threadIdx.x == 0 && s.gfix_n) *s.gfix_n = 0;
    if ((int)blockIdx.x >= nbi) {
        const int b = (blockIdx.x - nbi) * FB + threadIdx.x;
        if (b < m.nb) boundary_face<MODEL>(P, m, s, b, wall_rank, coef);
        return;
    }
    __shared__ double4 sw[WIN], sgx[WIN], sgy[WIN], sph[WIN];
    __shared__ double st[WIN];
    const int nc = m.nc;
    const int f0 = blockIdx.x * FB;
    const int f = f0 + threadIdx.x;
    const int2 e0 = m.fe[f0];
    const int base = min(e0.x, e0.y);
    // order and viscosity are shared by every solve of a pack
    const bool o2 = P[0].order == 2, grad = o2 || P[0].visc;
    for (int i = threadIdx.x; i < WIN; i += FB) {
        const int c = base + i;
        if (c < nc) {
            sw[i] = s.W4[c];
            st[i] = s.WT[c];
            if (grad) {
                sgx[i] = s.G4x[c];
                sgy[i] = s.G4y[c];
            }
            if (o2) sph[i] = s.PH4[c];
        }
    }
    __syncthreads();
    if (f >= m.nf) return;
    const int2 e = m.fe[f];
    const int sid = cell_solve(s, e.x);
    const Prm& p = P[sid];
    if (halted_behind(p, s.sc + sid)) return;
    const double4 z4 = make_double4(0.0, 0.0, 0.0, 0.0);
    const unsigned i0 = (unsigned)(e.x - base), i1 = (unsigned)(e.y - base);
    const bool in0 = i0 < (unsigned)WIN, in1 = i1 < (unsigned)WIN;
    const double4 w0 = in0 ? sw[i0] : s.W4[e.x], w1 = in1 ? sw[i1] : s.W4[e.y];
    const double t0 = in0 ? st[i0] : s.WT[e.x], t1 = in1 ? st[i1] : s.WT[e.y];
    double4 gx0 = z4, gy0 = z4, gx1 = z4, gy1 = z4, ph0 = z4, ph1 = z4;
    if (grad) {
        gx0 = in0 ? sgx[i0] : s.G4x[e.x];
        gy0 = in0 ? sgy[i0] : s.G4y[e.x];
        gx1 = in1 ? sgx[i1] : s.G4x[e.y];
        gy1 = in1 ? sgy[i1] : s.G4y[e.y];
    }
    if (o2) {
        ph0 = in0 ? sph[i0] : s.PH4[e.x];
        ph1 = in1 ? sph[i1] : s.PH4[e.y];
    }
    interior_face<MODEL>(p, m, s, f, e, w0, t0, gx0, gy0, ph0, w1, t1, gx1, gy1, ph1);
}

// Sum of the signed face fluxes of one cell in the reference's order (inter, then boundary, then the
// axisymmetric pressure source interAxisPressure, solver.c:646-683).
template <int MODEL>
__device__ __forceinline__ void gather_residual(const Prm& p, const Mesh& m, const State& s, int c, const double* P,
                                                double* R)
{
    constexpr int NV = Model<MODEL>::NV;
    const int nc = m.nc, nft = m.nf + m.nb;
#pragma unroll
    for (int k = 0; k < NV; k++) R[k] = 0.0;
    const int ns = m.nslot[c];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (j < ns) {
            int sf = m.fslot[(size_t)j * nc + c];
            int fi = sf > 0 ? sf - 1 : -sf - 1;
            double4 F = s.F4[fi];
            double fv[NV];
            fv[0] = F.x; fv[1] = F.y; fv[2] = F.z; fv[3] = F.w;
#pragma unroll
            for (int k = 4; k < NV; k++) fv[k] = s.Fx[(size_t)(k - 4) * nft + fi];
            if (sf > 0) {
#pragma unroll
                for (int k = 0; k < NV; k++) R[k] += fv[k];
            } else {
#pragma unroll
                for (int k = 0; k < NV; k++) R[k] -= fv[k];
            }
        }
    }
    if (p.axi == 1) {
        double dS = m.dslat[c];
        R[2] -= P[3] * dS;
        if constexpr (MODEL == 2) R[2] -= (2. / 3.) * P[0] * P[5] * dS;
    }
    if (p.laminar == 1 || MODEL >= 1) {
        // laminarInter / saInter face gather (laminar.c:77-98, sa.c:197-220), the SA source (sa.c:224-256),
        // then laminarBoundary / saBoundary (laminar.c:101-125, sa.c:351-368, 695-701)
        const int ni = m.nint[c];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (j < ni) {
                int sf = m.fslot[(size_t)j * nc + c];
                int fi = sf > 0 ? sf - 1 : -sf - 1;
                double4 V = s.FV[fi];
                if (sf > 0) {
                    R[1] -= V.x;
                    R[2] -= V.y;
                    R[3] -= V.z;
                    if constexpr (MODEL >= 1) R[4] -= V.w;
                    if constexpr (MODEL == 2) R[5] -= s.FV5[fi];
                } else {
                    R[1] += V.x;
                    R[2] += V.y;
                    R[3] += V.z;
                    if constexpr (MODEL >= 1) R[4] += V.w;
                    if constexpr (MODEL == 2) R[5] += s.FV5[fi];
                }
            }
        }
        if constexpr (MODEL == 1) {
            double4 gx = s.G4x[c], gy = s.G4y[c];
            double rho = P[0], T = P[4], n = P[5];
            double d = m.wall_d[c];
            double mi_L = sutherland(T);
            double n_L = mi_L / rho;
            double S = fabs(gy.y - gx.z);
            double Qt = p.sa_cc ? sacc_source(n, n_L, S, d, rho, gx.x, gy.x, s.Gxx[c], s.Gxy[c])
                                : sa_source(n, n_L, S, d, rho, gx.x, gy.x, s.Gxx[c], s.Gxy[c]);
            R[4] -= Qt * m.omega[c];
        }
        if constexpr (MODEL == 2) {
            double4 gx = s.G4x[c], gy = s.G4y[c];
            double sgx[4] = {gx.y, gx.z, s.Gxx[c], s.Gxx[(size_t)nc + c]};
            double sgy[4] = {gy.y, gy.z, s.Gxy[c], s.Gxy[(size_t)nc + c]};
            double Qtk, Qto;
            sst_cell_source(p.sst_k, sgx, sgy, P, m.wall_d[c], &Qtk, &Qto);
            if (P[6] != 0.0) {
                R[4] -= Qtk * m.omega[c];
                R[5] -= Qto * m.omega[c];
            }
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (j >= ni && j < ns) {
                int fi = m.fslot[(size_t)j * nc + c] - 1;
                double4 V = s.FV[fi];
                R[1] -= V.x;
                R[2] -= V.y;
                R[3] -= V.z;
                if constexpr (MODEL >= 1) R[4] -= V.w;
                if constexpr (MODEL == 2) R[5] -= s.FV5[fi];
            }
        }
    }
}

template <int MODEL>
__device__ __forceinline__ void storeR(const State& s, int nc, int c, const double* R)
{
    s.R4[c] = make_double4(R[0], R[1], R[2], R[3]);
#pragma unroll
    for (int k = 4; k < Model<MODEL>::NV; k++) s.Rx[(size_t)(k - 4) * nc + c] = R[k];
}

// the block's sum of R^2 per variable into s.part[blockIdx.x]: one row per cell block of NT cells (k_finalize
// is told how many rows a BLOCK-cell block has)
template <int MODEL, int NT = BLOCK>
__device__ __forceinline__ void partial_norms(const State& s, bool valid, const double* R)
{
    constexpr int NV = Model<MODEL>::NV;
    __shared__ double sh[NV][NT / 32];
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = valid ? R[k] * R[k] : 0.0;
    block_sum<NV, NT>(v, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < NV; k++) s.part[(size_t)blockIdx.x * NV + k] = v[k];
}

// The same partial sums one row per warp (32 cells, row = cell / 32), whatever the block size of the
// kernel: the rows, and so the norms summed from them, do not depend on the launch shape.
template <int MODEL>
__device__ __forceinline__ void partial_norms_warp(const State& s, bool valid, const double* R, int c)
{
    constexpr int NV = Model<MODEL>::NV;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        const double x = warp_sum(valid ? R[k] * R[k] : 0.0);
        if (lane == 0) s.part[(size_t)(c >> 5) * NV + k] = x;
    }
}

// ------------------------------------------------------------------------------------------------
// k_resid: R only (csu_residual).
// ------------------------------------------------------------------------------------------------
template <int MODEL>
__global__ void __launch_bounds__(BLOCK) k_resid(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                 const __grid_constant__ State s)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    const Prm& p = P[block_solve(s)];
    int c = blockIdx.x * BLOCK + threadIdx.x;
    bool valid = cell_in(p, c);
    double R[NV];
    if (valid) {
        double W[NP];
        loadP<MODEL>(s, m.nc, c, W);
        gather_residual<MODEL>(p, m, s, c, W, R);
        storeR<MODEL>(s, m.nc, c, R);
    }
    partial_norms<MODEL>(s, valid, R);
}

// ------------------------------------------------------------------------------------------------
// k_rk: one RK stage update (solverRK, solver.c:741-766) fused with the next residual's primitives.
// LAST: the stage that ends the iteration -- stores the state, the next local steps (solverCalcDt on the
// new, unclamped state) and the residual-norm partial sums of this stage's R (solverCalcRes).
// ------------------------------------------------------------------------------------------------
template <int MODEL, bool LAST>
__global__ void __launch_bounds__(BLOCK) k_rk(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                              const __grid_constant__ State s, double a)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    const int sid = block_solve(s);
    const Prm& p = P[sid];
    Scalars* const sc = s.sc + sid;
    if (halted(sc)) return;
    int c = blockIdx.x * BLOCK + threadIdx.x;
    bool valid = cell_in(p, c);
    double R[NV];
    double lmin = bitsd(0x7ff0000000000000ULL);
    if (valid) {
        double P[NP], U[NV];
        loadP<MODEL>(s, m.nc, c, P);
        gather_residual<MODEL>(p, m, s, c, P, R);
        loadU<MODEL>(s, m.nc, c, U);
        double om = m.omega[c];
        double dt = sc->dt_local == 1 ? s.dtl[c] : sc->dt;
#pragma unroll
        for (int k = 0; k < NV; k++) U[k] = U[k] - dt * p.sigma * a * R[k] / om;
        if (LAST) {
            double l = local_step<MODEL>(p, U, m.sxh[c], m.syh[c], om);
            s.dtl[c] = cfl_at(p, sc->iter + 1) * l;
            lmin = l;
            clamp_prim<MODEL>(p, U, P);
            storeU<MODEL>(s, m.nc, c, U);
            storeR<MODEL>(s, m.nc, c, R);
        } else {
            clamp_prim<MODEL>(p, U, P);
        }
        storeP<MODEL>(s, m.nc, c, P);
    }
    if (LAST) {
        double v = block_min(lmin);
        if (threadIdx.x == 0 && !(v > bitsd(0x7fefffffffffffffULL))) atomicMin(&sc->dtmin_bits, dbits(v));
        partial_norms<MODEL>(s, valid, R);
    }
}

// implicitAuxCalcFlux2 (implicit.c:183-191) and its _sa/_sst forms
template <int NV>
__device__ __forceinline__ void aux_flux(const double* U, double pr, double nx, double ny, double* F)
{
    double V = (nx * U[1] + ny * U[2]) / U[0];
    F[0] = U[0] * V;
    F[1] = U[1] * V + nx * pr;
    F[2] = U[2] * V + ny * pr;
    F[3] = (U[3] + pr) * V;
#pragma unroll
    for (int k = 4; k < NV; k++) F[k] = U[k] * V;
}

// ------------------------------------------------------------------------------------------------
// k_impl: R (WITH_R) and the implicit diagonal (implicitCalcD, implicit.c:19-181) of each cell. The
// diagonal, the local steps and their minimum need only the iteration's start state, so DPLUR computes them
// beside the gradient and flux kernels and gathers R in its first sweep.
// ------------------------------------------------------------------------------------------------
template <int MODEL, bool WITH_R>
__global__ void __launch_bounds__(BLOCK) k_impl(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                const __grid_constant__ State s)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    const int sid = block_solve(s);
    const Prm& p = P[sid];
    Scalars* const sc = s.sc + sid;
    if (halted(sc)) return;
    int c = blockIdx.x * BLOCK + threadIdx.x;
    bool valid = cell_in(p, c);
    double R[NV];
    double lmin = bitsd(0x7ff0000000000000ULL);
    if (valid) {
        const int nc = m.nc;
        double P[NP];
        loadP<MODEL>(s, nc, c, P);
        if (WITH_R) {
            gather_residual<MODEL>(p, m, s, c, P, R);
            storeR<MODEL>(s, nc, c, R);
        }
        {
            if constexpr (MODEL == 1) {
                // extension (saImplicitSource): the SA source's derivative in rho nt by a forward difference
                // in nt (the gradients held), its negative (destruction-dominated) part taken implicitly:
                // dQ = -Omega min(dQt/d(rho nt), 0) >= 0 joins the diagonal of the nt row
                if (p.sa_isrc) {
                    double4 gx = s.G4x[c], gy = s.G4y[c];
                    double rho = P[0], T = P[4], n = P[5];
                    double d = m.wall_d[c];
                    double mi_L = sutherland(T);
                    double n_L = mi_L / rho;
                    double S = fabs(gy.y - gx.z);
                    double hn = 1e-6 * fmax(fabs(n), n_L);
                    double q0 = p.sa_cc ? sacc_source(n, n_L, S, d, rho, gx.x, gy.x, s.Gxx[c], s.Gxy[c])
                                        : sa_source(n, n_L, S, d, rho, gx.x, gy.x, s.Gxx[c], s.Gxy[c]);
                    double q1 = p.sa_cc ? sacc_source(n + hn, n_L, S, d, rho, gx.x, gy.x, s.Gxx[c], s.Gxy[c])
                                        : sa_source(n + hn, n_L, S, d, rho, gx.x, gy.x, s.Gxx[c], s.Gxy[c]);
                    double dq = (q1 - q0) / hn / rho;
                    s.dQ[c] = isfinite(dq) ? -m.omega[c] * fmin(dq, 0.0) : 0.0;
                }
            }
            if constexpr (MODEL == 2) {
                // the SST source Jacobians of the implicit diagonal (sstInterSource, sst.c:643-680): LU-SGS
                // as the reference, DPLUR as the extension's k-omega diagonal block
                if (s.dQ) {
                    double4 gx = s.G4x[c], gy = s.G4y[c];
                    double sgx[4] = {gx.y, gx.z, s.Gxx[c], s.Gxx[(size_t)nc + c]};
                    double sgy[4] = {gy.y, gy.z, s.Gxy[c], s.Gxy[(size_t)nc + c]};
                    double J[6];
                    sst_source_jacobians(p.sst_k, sgx, sgy, P, m.wall_d[c], m.omega[c], J);
#pragma unroll
                    for (int q = 0; q < 6; q++) s.dQ[(size_t)q * nc + c] = J[q];
                }
            }
        }
        const int ni = m.nint[c], ns = m.nslot[c];
        double Lc = 0, Lv = 0;
        for (int j = 0; j < ni; j++) {
            int sf = m.fslot[(size_t)j * nc + c];
            int f = sf > 0 ? sf - 1 : -sf - 1;
            int2 e = m.fe[f];
            double4 w0 = s.W4[e.x], w1 = s.W4[e.y];
            double T0 = s.WT[e.x], T1 = s.WT[e.y];
            double2 dSv = m.fn[f];
            double dS = m.fds[f];
            double u = (w0.y + w1.y) * 0.5;
            double v = (w0.z + w1.z) * 0.5;
            double T = (T0 + T1) * 0.5;
            double cc = T2c(p.gas, T);
            double nx = dSv.x / dS, ny = dSv.y / dS;
            Lc += (fabs(nx * u + ny * v) + cc) * dS;
            if constexpr (MODEL >= 1) {
                double r = (w0.x + w1.x) * 0.5;
                double mi = sutherland(T);
                Lv += fmax(4 / (3 * r), T2gamma(p.gas, T) / r) * (mi / p.pr + s.MIT[f] / p.pr_t) * dS * dS;
            } else if (p.laminar) {
                double r = (w0.x + w1.x) * 0.5;
                Lv += visc_radius(p.gas, p.pr, r, T) * dS * dS;
            }
        }
        double D = 0.5 * p.w_imp * Lc;
        if (p.visc) D += Lv / m.omega[c];
        for (int j = ni; j < ns; j++) {
            int b = m.fslot[(size_t)j * nc + c] - 1 - m.nf;
            double2 dSv = m.bn[b];
            double dS = m.bds[b];
            double cc = T2c(p.gas, P[4]);
            double nx, ny;
            if (dS > 0) {
                nx = dSv.x / dS;
                ny = dSv.y / dS;
            } else {
                nx = 0.0;
                ny = 1.0;
            }
            double Lb = (fabs(nx * P[1] + ny * P[2]) + cc) * dS;
            Lc += Lb;
            D += 0.5 * p.w_imp * Lb;
            if (p.visc) {
                double Lvb = visc_radius(p.gas, p.pr, P[0], P[4]) * dS * dS;
                D += Lvb / m.omega[c];
            }
        }
        double om = m.omega[c];
        double l = om / Lc;
        s.dtl[c] = l;
        s.dpart[c] = D;
        lmin = l;
    }
    double v = block_min(lmin);
    if (threadIdx.x == 0 && !(v > bitsd(0x7fefffffffffffffULL))) atomicMin(&sc->dtmin_bits, dbits(v));
    if (WITH_R) partial_norms<MODEL>(s, valid, R);
}

// ------------------------------------------------------------------------------------------------
// k_face_mit: the SA face eddy viscosity mu_t = fv1 rho nt of the face means of the two cells' primitives
// (saBoundaryVisc's interior part, sa.c: the same expressions as sa_face_flux / sacc_face_flux, whose value
// it equals bit for bit), for the DPLUR blocks and diagonal: it needs no gradient, so they can run beside
// k_grad and k_flux instead of after them.
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(BLOCK) k_face_mit(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                    const __grid_constant__ State s)
{
    const int f = blockIdx.x * BLOCK + threadIdx.x;
    if (f >= m.nf) return;
    const int2 e = m.fe[f];
    const int sid = cell_solve(s, e.x);
    if (halted(s.sc + sid)) return;
    const int nc = m.nc;
    const double4 w0 = s.W4[e.x], w1 = s.W4[e.y];
    const double r = (w1.x + w0.x) * 0.5;
    const double T = (s.WT[e.y] + s.WT[e.x]) * 0.5;
    const double n = (s.Wx[e.y] + s.Wx[e.x]) * 0.5;
    const double mi_L = sutherland(T);
    const double n_L = mi_L / r;
    double fv1, tx, ty;
    sa_face(n, n_L, r, 0.0, 0.0, &fv1, &tx, &ty);
    s.MIT[f] = fv1 * r * n;
    (void)nc;
}

// ------------------------------------------------------------------------------------------------
// k_blocks: the DPLUR off-diagonal blocks of implicitUpdateA (implicit.c:689-813; implicitUpdateA_sa
// 860-935), one thread per interior face slot j of a cell: the finite-difference Jacobian (h = 1e-6) of the
// neighbour's face flux, minus half the face's spectral radius on the diagonal. A block needs only the
// state at the start of the iteration (and, for SA, the face eddy viscosity of k_flux), so the engine runs
// this kernel beside the gradient and flux kernels. Blocks [j gb, (j + 1) gb) of the grid hold slot j of
// the cells of cell blocks [0, gb).
// ------------------------------------------------------------------------------------------------
template <int MODEL>
__global__ void __launch_bounds__(BLOCK, MODEL == 0 ? 3 : 2) k_blocks(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                  const __grid_constant__ State s, int gb)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    const int j = blockIdx.x / gb, cb = blockIdx.x - j * gb;
    const int sid = s.bsolve ? s.bsolve[cb] : 0;
    const Prm& p = P[sid];
    const Scalars* const sc = s.sc + sid;
    if (halted(sc)) return;
    const int c = cb * BLOCK + threadIdx.x;
    if (!cell_in(p, c)) return;
    const int nc = m.nc;
    if (j >= m.nint[c]) return;
    const int sf = m.fslot[(size_t)j * nc + c];
    const int f = sf > 0 ? sf - 1 : -sf - 1;
    const int2 e = m.fe[f];
    const int nb = sf > 0 ? e.y : e.x;
    const double2 dSv = m.fn[f];
    const double dSx = sf > 0 ? dSv.x : -dSv.x, dSy = sf > 0 ? dSv.y : -dSv.y;
    const double dS = m.fds[f];
    const double nx = dSx / dS, ny = dSy / dS;
    const double h = 1.0e-6;
    double Un[NV], Pn[NP];
    loadU<MODEL>(s, nc, nb, Un);
    loadP<MODEL>(s, nc, nb, Pn);
    double F0[NV], F[NV], Uq[NV];
    double rho = Un[0];
    double uu = Un[1] / rho;
    double vv = Un[2] / rho;
    double E = Un[3] / rho;
    aux_flux<NV>(Un, Pn[3], nx, ny, F0);
    double ee0 = E - 0.5 * (uu * uu + vv * vv);
    // SST (an extension: the reference's SST DPLUR multiplies 4x4 blocks into six variables, implicit.c:
    // 990-1000 with 938-972): the energy holds the turbulent kinetic energy, as in its SST delta flux
    // (implicitCalcDeltaFlux_sst, implicit.c:1048-1118)
    if constexpr (MODEL == 2) ee0 = ee0 - Un[4] / rho;
    double A[NV * NV];
#pragma unroll
    for (int mm = 0; mm < NV; mm++) {
        // SST: rho omega reaches 1e10 beside a wall, where a step of 1e-6 is below its last bit; its column
        // (a flux linear in rho omega) takes a step relative to the value
        const double hm = MODEL == 2 && mm >= 4 ? h * fmax(1.0, fabs(Un[mm])) : h;
#pragma unroll
        for (int nn = 0; nn < NV; nn++) Uq[nn] = mm == nn ? Un[nn] + hm : Un[nn];
        double r2 = Uq[0];
        double u2 = Uq[1] / r2;
        double v2 = Uq[2] / r2;
        double E2 = Uq[3] / r2;
        double ee1 = E2 - 0.5 * (u2 * u2 + v2 * v2);
        if constexpr (MODEL == 2) ee1 = ee1 - Uq[4] / r2;
        double T = e2Taprox(p.gas, ee0, Pn[4], ee1);
        double pr = p.gas.R * r2 * T;
        aux_flux<NV>(Uq, pr, nx, ny, F);
#pragma unroll
        for (int nn = 0; nn < NV; nn++) A[nn * NV + mm] = 0.5 * (F[nn] - F0[nn]) * dS / hm;
    }
    double cc = T2c(p.gas, Pn[4]);
    double ra = p.w_imp * (fabs(nx * Pn[1] + ny * Pn[2]) + cc) * dS;
    if constexpr (MODEL >= 1) {
        // implicitUpdateA_sa (implicit.c:920-928): always viscous, with the face eddy viscosity (SST: the
        // same radius with its own eddy viscosity)
        double Pc[NP];
        loadP<MODEL>(s, nc, c, Pc);
        double r = (Pc[0] + Pn[0]) * 0.5;
        double T = (Pc[4] + Pn[4]) * 0.5;
        double mi = sutherland(T);
        ra += fmax(4 / (3 * r), T2gamma(p.gas, T) / r) * (mi / p.pr + s.MIT[f] / p.pr_t) * dS / m.fL[f];
    } else if (p.laminar) {
        double Pc[NP];
        loadP<MODEL>(s, nc, c, Pc);
        double r = (Pc[0] + Pn[0]) * 0.5;
        double T = (Pc[4] + Pn[4]) * 0.5;
        ra += visc_radius(p.gas, p.pr, r, T) * dS / m.fL[f];
    }
#pragma unroll
    for (int nn = 0; nn < NV; nn++) A[nn * NV + nn] -= 0.5 * ra;
    const size_t base = (size_t)j * NV * NV * nc + c;
    if (p.blk32) {
#pragma unroll
        for (int q = 0; q < NV * NV; q++) s.blocks32[base + (size_t)q * nc] = (float)A[q];
    } else {
#pragma unroll
        for (int q = 0; q < NV * NV; q++) s.blocks[base + (size_t)q * nc] = A[q];
    }
}

// ------------------------------------------------------------------------------------------------
// k_sweep: one relaxed Jacobi sweep of implicitCalcDPLUR (implicit.c:1006-1033, implicitMultA 938-972):
//   x_new = w (-R - (D x + sum_j A_j x_j)) / D + x,  w = 2/3,  D += Omega/dt with dt = CFL min(Omega/Lc).
// The early exit of the reference (max |dx_0| < 1e-14 after a sweep) is taken on the device: a sweep that
// finds the previous one converged copies x forward. LAST adds the increment to the state
// (solverUpdateUImplicit, solver.c:1945-1955) and computes the next iteration's primitives. FIRST gathers
// the cell's residual R from the face fluxes (as k_impl does), stores it for the later sweeps and writes
// the block's partial norms.
// ------------------------------------------------------------------------------------------------
template <int MODEL, bool LAST, bool FIRST, int SB, bool F32>
__global__ void __launch_bounds__(SB) k_sweep(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                              const __grid_constant__ State s, int sweep, int cur)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    static_assert(BLOCK % SB == 0, "sweep blocks tile the cell blocks");
    // SB-thread blocks: BLOCK / SB of them cover one cell block of the solve map
    const int sid = s.bsolve ? s.bsolve[blockIdx.x / (BLOCK / SB)] : 0;
    const Prm& p = P[sid];
    Scalars* const sc = s.sc + sid;
    if (halted(sc)) return;
    int c = blockIdx.x * SB + threadIdx.x;
    const int nc = m.nc;
    bool conv = !FIRST && sweep > 0 && bitsd(sc->sweep_max[sweep - 1]) < 1e-14;
    double dmax = 0.0;
    const bool valid = cell_in(p, c);
    double R[NV];
    if (valid) {
        const double4* xo4 = s.X4[cur];
        const double* xox = s.Xx[cur];
        double4* xn4 = s.X4[cur ^ 1];
        double* xnx = s.Xx[cur ^ 1];
        double xo[NV], xn[NV];
        {
            double4 t = xo4[c];
            xo[0] = t.x; xo[1] = t.y; xo[2] = t.z; xo[3] = t.w;
#pragma unroll
            for (int k = 4; k < NV; k++) xo[k] = xox[(size_t)(k - 4) * nc + c];
        }
        if constexpr (FIRST) {
            double Pc[NP];
            loadP<MODEL>(s, nc, c, Pc);
            gather_residual<MODEL>(p, m, s, c, Pc, R);
            storeR<MODEL>(s, nc, c, R);
        } else {
            double4 t = s.R4[c];
            R[0] = t.x; R[1] = t.y; R[2] = t.z; R[3] = t.w;
#pragma unroll
            for (int k = 4; k < NV; k++) R[k] = s.Rx[(size_t)(k - 4) * nc + c];
        }
        if (conv) {
#pragma unroll
            for (int k = 0; k < NV; k++) xn[k] = xo[k];
        } else {
            double cfl = cfl_at(p, sc->iter);
            double dt = p.implicit_local_dt ? s.dtl[c] * cfl : bitsd(sc->dtmin_bits) * cfl;
            double D = s.dpart[c] + m.omega[c] / dt;
            // y = D x + sum_j A_j x_j; SST keeps the off-diagonal sum alone (its diagonal is a block)
            double y[NV];
#pragma unroll
            for (int k = 0; k < NV; k++) y[k] = MODEL == 2 ? 0.0 : D * xo[k];
            // SA with saImplicitSource: the nt row's diagonal also holds the implicit source part
            double D4 = D;
            if constexpr (MODEL == 1) {
                if (p.sa_isrc) {
                    D4 = D + s.dQ[c];
                    y[4] = D4 * xo[4];
                }
            }
            // Slots 0-2 are gathered unconditionally (a slot without a face reads the cell itself and a zero
            // block, both in bounds, and is not summed), so their index and neighbour loads issue together
            // instead of one dependent chain per face; slot 3 only exists in quadrilaterals.
            const int ni = m.nint[c];
            int nbj[4];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                int q = m.fnb[(size_t)j * nc + c];
                nbj[j] = q >= 0 ? q : c;
            }
            nbj[3] = ni > 3 ? m.fnb[(size_t)3 * nc + c] : c;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (j == 3 && ni <= 3) break;
                const int nb = nbj[j];
                double xb[NV];
                double4 t = xo4[nb];
                xb[0] = t.x; xb[1] = t.y; xb[2] = t.z; xb[3] = t.w;
#pragma unroll
                for (int k = 4; k < NV; k++) xb[k] = xox[(size_t)(k - 4) * nc + nb];
                const size_t base = (size_t)j * NV * NV * nc + c;
                const bool use = j < ni;
                if constexpr (F32) {
                    // FP32 blocks kept as floats until they are used: fewer registers, more cells in flight
                    float Af[NV * NV];
#pragma unroll
                    for (int q = 0; q < NV * NV; q++) Af[q] = s.blocks32[base + (size_t)q * nc];
                    if (use) {
#pragma unroll
                        for (int kk = 0; kk < NV; kk++)
#pragma unroll
                            for (int nn = 0; nn < NV; nn++) y[kk] += (double)Af[kk * NV + nn] * xb[nn];
                    }
                } else {
                    // FP64 blocks (the FP32 branch stays for contexts launched without F32: as compiled with
                    // it, the FP64 sweep keeps more of its loads in flight than an FP64-only build does)
                    double A[NV * NV];
                    if (p.blk32) {
#pragma unroll
                        for (int q = 0; q < NV * NV; q++) A[q] = (double)s.blocks32[base + (size_t)q * nc];
                    } else {
#pragma unroll
                        for (int q = 0; q < NV * NV; q++) A[q] = s.blocks[base + (size_t)q * nc];
                    }
                    if (use) {
#pragma unroll
                        for (int kk = 0; kk < NV; kk++)
#pragma unroll
                            for (int nn = 0; nn < NV; nn++) y[kk] += A[kk * NV + nn] * xb[nn];
                    }
                }
            }
            const double w = 2. / 3.;
            if constexpr (MODEL == 2) {
                // SST (extension): D on the mean flow; on k and omega, D minus the non-positive (destruction)
                // part of the source Jacobians' diagonal, with their coupling to rho (the LU-SGS diagonal
                // block, implicit.c:323-345, without its production part and k-omega cross terms, which made
                // the iteration diverge at CFL 2 on wall-resolved meshes): x* = Dblock^-1 (-R - sum_j A_j x_j),
                // then x += w (x* - x)
                double z[NV], xs[NV];
#pragma unroll
                for (int k = 0; k < NV; k++) z[k] = -R[k] - y[k];
#pragma unroll
                for (int k = 0; k < 4; k++) xs[k] = z[k] / D;
                const double a = D - fmin(s.dQ[(size_t)nc + c], 0.0);
                const double dq = D - fmin(s.dQ[(size_t)5 * nc + c], 0.0);
                xs[4] = (z[4] + s.dQ[c] * xs[0]) / a;
                xs[5] = (z[5] + s.dQ[(size_t)3 * nc + c] * xs[0]) / dq;
#pragma unroll
                for (int k = 0; k < NV; k++) xn[k] = xo[k] + w * (xs[k] - xo[k]);
            } else {
#pragma unroll
                for (int k = 0; k < NV; k++) xn[k] = w * (-R[k] - y[k]) / (k == 4 ? D4 : D) + xo[k];
            }
            dmax = fabs(xn[0] - xo[0]);
        }
        xn4[c] = make_double4(xn[0], xn[1], xn[2], xn[3]);
#pragma unroll
        for (int k = 4; k < NV; k++) xnx[(size_t)(k - 4) * nc + c] = xn[k];
        if (LAST) {
            double U[NV], P[NP];
            loadU<MODEL>(s, nc, c, U);
#pragma unroll
            for (int k = 0; k < NV; k++) U[k] += xn[k];
            clamp_prim<MODEL>(p, U, P);
            storeU<MODEL>(s, nc, c, U);
            storeP<MODEL>(s, nc, c, P);
        }
    }
    if (!conv) {
        double v = block_max<SB>(dmax);
        if (threadIdx.x == 0) atomicMax(&sc->sweep_max[sweep], dbits(v));
    }
    if (FIRST) partial_norms_warp<MODEL>(s, valid, R, c);
}

// implicitCalcDeltaFlux (implicit.c:194-231) and implicitCalcDeltaFlux_sa (495-552): F(U + d) - F(U) on the
// face normal, from the neighbour's primitives P and increment d.
template <int MODEL>
__device__ __forceinline__ void delta_flux(const Prm& p, const double* P, const double* d, double nx, double ny,
                                           double* dF)
{
    constexpr int NV = Model<MODEL>::NV;
    double rho = P[0], u = P[1], v = P[2], pr = P[3];
    double U[NV], F0[NV], F1[NV];
    double T = pr / (p.gas.R * rho);
    double e0 = T2e(p.gas, T);
    double E = e0 + (u * u + v * v) / 2;
    if constexpr (MODEL == 2) E = E + P[5]; // implicitCalcDeltaFlux_sst (implicit.c:1048-1118): + k
    U[0] = rho;
    U[1] = rho * u;
    U[2] = rho * v;
    U[3] = rho * E;
    if constexpr (MODEL >= 1) U[4] = rho * P[5];
    if constexpr (MODEL == 2) U[5] = rho * P[6];
    aux_flux<NV>(U, pr, nx, ny, F0);
#pragma unroll
    for (int k = 0; k < NV; k++) U[k] = U[k] + d[k];
    if constexpr (MODEL == 0) {
        rho = U[0];
        u = U[1] / rho;
        v = U[2] / rho;
        E = U[3] / rho;
        double e1 = E - 0.5 * (u * u + v * v);
        T = e2Taprox(p.gas, e0, T, e1);
        pr = p.gas.R * T * rho;
    } else if constexpr (MODEL == 2) {
        rho = U[0];
        rho = fmax(rho, p.r_lim);
        U[0] = rho;
        u = U[1] / rho;
        v = U[2] / rho;
        double k = U[4] / rho;
        if (k < 1e-14) {
            k = 1e-14;
            U[4] = rho * k;
        }
        double om = U[5] / rho;
        if (om < 0.0) { // omLim = 0 (solver.c:1155)
            om = 0.0;
            U[5] = rho * om;
        }
        E = U[3] / rho;
        double e1 = E - (u * u + v * v) * 0.5 - k;
        e1 = fmax(e1, 7.176325e+02);
        T = e2Taprox(p.gas, e0, T, e1);
        if (T < 1) {
            T = 1;
            e1 = T2e(p.gas, T);
            E = e1 + (u * u + v * v) * 0.5 + k;
            U[3] = rho * E;
        }
        pr = p.gas.R * T * rho;
    } else {
        rho = U[0];
        rho = fmax(rho, p.r_lim);
        U[0] = rho;
        u = U[1] / rho;
        v = U[2] / rho;
        E = U[3] / rho;
        double e1 = E - (u * u + v * v) * 0.5;
        e1 = fmax(e1, 7.176325e+02);
        T = e2Taprox(p.gas, e0, T, e1);
        if (T < 1) {
            T = 1;
            e1 = T2e(p.gas, T);
            E = e1 + (u * u + v * v) * 0.5;
            U[3] = rho * E;
        }
        pr = p.gas.R * T * rho;
        double n = U[4] / rho;
        n = fmax(n, 0);
        U[4] = rho * n;
    }
    aux_flux<NV>(U, pr, nx, ny, F1);
#pragma unroll
    for (int k = 0; k < NV; k++) dF[k] = F1[k] - F0[k];
}

// ------------------------------------------------------------------------------------------------
// k_lusgs: one colour of the LU-SGS sweeps (implicitLUSGS_L / _U, implicit.c:274-482) as a multicolour
// Gauss-Seidel: the reference sweeps cells in index order using the already-updated lower (upper) index
// neighbours; here the cells of one colour update together using the neighbours of lower (higher) colours.
// Same operator, another ordering: the converged solution is the same, the path to it is not.
//   FWD: x0_i = (-R_i - sum_{lower} 0.5 (dF(x0_j) dS - ra_j x0_j)) / D_i
//   BWD: x1_i = (D_i x0_i - sum_{higher} 0.5 (dF(x1_j) dS - ra_j x1_j)) / D_i
// ------------------------------------------------------------------------------------------------
template <int MODEL, bool FWD>
__global__ void __launch_bounds__(BLOCK) k_lusgs(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                 const __grid_constant__ State s, const int* color,
                                                 const int* cells, int mycolor, int start, int count)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    int t = blockIdx.x * BLOCK + threadIdx.x;
    if (t >= count) return;
    const int nc = m.nc;
    int c = cells[start + t];
    const int sid = cell_solve(s, c);
    const Prm& p = P[sid];
    Scalars* const sc = s.sc + sid;
    if (halted(sc)) return;
    const double4* src4 = FWD ? s.X4[0] : s.X4[1];
    const double* srcx = FWD ? s.Xx[0] : s.Xx[1];
    double cfl = cfl_at(p, sc->iter);
    double dt = p.implicit_local_dt ? s.dtl[c] * cfl : bitsd(sc->dtmin_bits) * cfl;
    double D = s.dpart[c] + m.omega[c] / dt;
    double x[NV];
    if (FWD) {
        double4 t4 = s.R4[c];
        x[0] = -t4.x; x[1] = -t4.y; x[2] = -t4.z; x[3] = -t4.w;
#pragma unroll
        for (int k = 4; k < NV; k++) x[k] = -s.Rx[(size_t)(k - 4) * nc + c];
    } else {
        double4 t4 = s.X4[0][c];
        x[0] = D * t4.x; x[1] = D * t4.y; x[2] = D * t4.z; x[3] = D * t4.w;
#pragma unroll
        for (int k = 4; k < NV; k++) x[k] = D * s.Xx[0][(size_t)(k - 4) * nc + c];
        if constexpr (MODEL == 2) {
            // implicitLUSGS_U (implicit.c:372-390): the k, omega rows multiply by the SST diagonal block
            const double x0 = t4.x, x4 = s.Xx[0][c], x5 = s.Xx[0][(size_t)nc + c];
            const double a = D - s.dQ[(size_t)nc + c], b = -s.dQ[(size_t)2 * nc + c];
            const double cq = -s.dQ[(size_t)4 * nc + c], dq = D - s.dQ[(size_t)5 * nc + c];
            const double det = a * dq - b * cq;
            if (!(fabs(det) < 1e-14)) {
                x[4] = a * x4 + b * x5 - s.dQ[c] * x0;
                x[5] = cq * x4 + dq * x5 - s.dQ[(size_t)3 * nc + c] * x0;
            }
        }
    }
    double P0[NP];
    loadP<MODEL>(s, nc, c, P0);
    const int ni = m.nint[c];
    for (int j = 0; j < ni; j++) {
        int sf = m.fslot[(size_t)j * nc + c];
        int f = sf > 0 ? sf - 1 : -sf - 1;
        int2 e = m.fe[f];
        int nb = sf > 0 ? e.y : e.x;
        int cn = color[nb];
        if (FWD ? (cn >= mycolor) : (cn <= mycolor)) continue;
        double2 dSv = m.fn[f];
        double dSx = sf > 0 ? dSv.x : -dSv.x, dSy = sf > 0 ? dSv.y : -dSv.y;
        double dS = m.fds[f];
        double nx = dSx / dS, ny = dSy / dS;
        double Pn[NP], dn[NV], dF[NV];
        loadP<MODEL>(s, nc, nb, Pn);
        {
            double4 t4 = src4[nb];
            dn[0] = t4.x; dn[1] = t4.y; dn[2] = t4.z; dn[3] = t4.w;
#pragma unroll
            for (int k = 4; k < NV; k++) dn[k] = srcx[(size_t)(k - 4) * nc + nb];
        }
        delta_flux<MODEL>(p, Pn, dn, nx, ny, dF);
        double cc = T2c(p.gas, Pn[4]);
        double ra = p.w_imp * (fabs(nx * Pn[1] + ny * Pn[2]) + cc) * dS;
        if constexpr (MODEL >= 1) {
            // implicitFunc_sa / implicitFunc_sst (implicit.c:560-567, 1140-1150): the face eddy viscosity
            double r = Pn[0], T = Pn[4];
            double mi = sutherland(T);
            ra += fmax(4 / (3 * r), T2gamma(p.gas, T) / r) * (mi / p.pr + s.MIT[f] / p.pr_t) * dS / m.fL[f];
        } else if (p.laminar) {
            ra += visc_radius(p.gas, p.pr, Pn[0], Pn[4]) * dS / m.fL[f];
        }
#pragma unroll
        for (int k = 0; k < NV; k++) x[k] -= 0.5 * (dF[k] * dS - ra * dn[k]);
    }
    if constexpr (MODEL == 2) {
        // the SST diagonal (implicit.c:323-345, 444-465): D on the mean flow, a 2x2 block with the source
        // Jacobians on k and omega, its determinant in double and the quotients in long double
#pragma unroll
        for (int k = 0; k < 4; k++) x[k] /= D;
        const double A = x[4] + s.dQ[c] * x[0];
        const double B = x[5] + s.dQ[(size_t)3 * nc + c] * x[0];
        const double a = D - s.dQ[(size_t)nc + c], b = -s.dQ[(size_t)2 * nc + c];
        const double cq = -s.dQ[(size_t)4 * nc + c], dq = D - s.dQ[(size_t)5 * nc + c];
        const double det = a * dq - b * cq;
        if (fabs(det) < 1e-14) {
            x[4] /= D;
            x[5] /= D;
        } else {
            const double n4 = A * dq - B * b, n5 = -A * cq + B * a;
            bool ok = true;
            const double q4 = x87_div_d(n4, det, ok);
            const double q5 = x87_div_d(n5, det, ok);
            if (ok) {
                x[4] = q4;
                x[5] = q5;
            } else {
                const X80 dx = x80_from_double(det);
                x[4] = x80_to_double(x80_div(x80_from_double(n4), dx));
                x[5] = x80_to_double(x80_div(x80_from_double(n5), dx));
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < NV; k++) x[k] /= D;
    }
    double4* dst4 = FWD ? s.X4[0] : s.X4[1];
    double* dstx = FWD ? s.Xx[0] : s.Xx[1];
    dst4[c] = make_double4(x[0], x[1], x[2], x[3]);
#pragma unroll
    for (int k = 4; k < NV; k++) dstx[(size_t)(k - 4) * nc + c] = x[k];
}

// U += dW1 (solverUpdateUImplicit), then the next iteration's primitives and clamps
template <int MODEL>
__global__ void __launch_bounds__(BLOCK) k_update(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                  const __grid_constant__ State s)
{
    constexpr int NV = Model<MODEL>::NV, NP = Model<MODEL>::NP;
    const Prm& p = P[block_solve(s)];
    if (halted(s.sc + block_solve(s))) return;
    int c = blockIdx.x * BLOCK + threadIdx.x;
    if (!cell_in(p, c)) return;
    const int nc = m.nc;
    double U[NV], W[NP];
    loadU<MODEL>(s, nc, c, U);
    double4 t4 = s.X4[1][c];
    U[0] += t4.x; U[1] += t4.y; U[2] += t4.z; U[3] += t4.w;
#pragma unroll
    for (int k = 4; k < NV; k++) U[k] += s.Xx[1][(size_t)(k - 4) * nc + c];
    clamp_prim<MODEL>(p, U, W);
    storeU<MODEL>(s, nc, c, U);
    storeP<MODEL>(s, nc, c, W);
}

// ------------------------------------------------------------------------------------------------
// k_finalize: one block closing an iteration (solverCalcRes, solverCalcCoeff3, history row, flags) and
// preparing the next step size. mode: 0 RK iteration, 1 implicit iteration, 2 prologue (step size only),
// 3 residual only (norms). bsel: the face-coefficient buffer k_flux wrote (0 bcoef, 1 bcoef2). In mode 1
// it records the halt flags it found on entry in `frozen` (halted_behind).
// ------------------------------------------------------------------------------------------------
template <int MODEL>
__global__ void __launch_bounds__(BLOCK) k_finalize(const Prm* __restrict__ P, const __grid_constant__ Mesh m,
                                                    const __grid_constant__ State s, int mode, int ppb, int bsel)
{
    constexpr int NV = Model<MODEL>::NV;
    __shared__ double sh[NV + 4][BLOCK / 32];
    const int sid = blockIdx.x; // one block per solve
    const Prm& p = P[sid];
    Scalars* const sc = s.sc + sid;
    // ppb rows of partial norms per cell block (the DPLUR first sweep writes one per 128 cells)
    const int npart = p.nblk * ppb, nwall = p.nwall;
    const double* part = s.part + (size_t)p.blk0 * ppb * NV;
    const double* bcoef = (bsel ? s.bcoef2 : s.bcoef) + (size_t)p.wall0 * 4;
    // Everything the block reads is requested before the halted test, so the loads overlap: a chain of
    // dependent round trips to the L2 would be most of a one-block kernel's time. Thread 0 keeps a copy of
    // the solve's scalars and writes back only what changes.
    const bool stop = mode != 2 && mode != 3 && halted(sc);
    double v[NV + 4];
#pragma unroll
    for (int k = 0; k < NV + 4; k++) v[k] = 0.0;
    if (mode != 2) {
        // rows strided over the threads (consecutive threads read consecutive rows), four rows per thread in
        // flight before any is added, then a fixed tree: deterministic
        constexpr int U = 4;
        for (int i0 = threadIdx.x; i0 < npart; i0 += U * BLOCK) {
            double t[U][NV];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int i = i0 + u * BLOCK;
#pragma unroll
                for (int k = 0; k < NV; k++) t[u][k] = i < npart ? part[(size_t)i * NV + k] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < U; u++)
#pragma unroll
                for (int k = 0; k < NV; k++) v[k] += t[u][k];
        }
        for (int i0 = threadIdx.x; i0 < nwall; i0 += U * BLOCK) {
            double t[U][4];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int i = i0 + u * BLOCK;
#pragma unroll
                for (int k = 0; k < 4; k++) t[u][k] = i < nwall ? bcoef[(size_t)i * 4 + k] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < U; u++)
#pragma unroll
                for (int k = 0; k < 4; k++) v[NV + k] += t[u][k];
        }
    }
    Scalars S;
    if (threadIdx.x == 0) {
        S = *sc;
        if (mode == 1) sc->frozen = stop;
    }
    if (stop) return;
    block_sum<NV + 4>(v, sh);
    if (threadIdx.x != 0) return;
    if (mode != 2) {
        bool bad = false;
        double res[NV];
        for (int k = 0; k < NV; k++) {
            res[k] = sqrt(v[k] / p.nc);
            sc->res[k] = res[k];
            if (!isfinite(res[k])) bad = true;
        }
        // Cx_v -= fx/q per wall face (solver.c:1376-1380): the negated sum
        double cxp = v[NV] / p.sref, cyp = v[NV + 1] / p.sref;
        double cxv = (0.0 - v[NV + 2]) / p.sref, cyv = (0.0 - v[NV + 3]) / p.sref;
        if (p.axi) {
            cxp *= 2 * M_PI;
            cxv *= 2 * M_PI;
        }
        sc->coef[0] = cxp; sc->coef[1] = cxv; sc->coef[2] = cyp; sc->coef[3] = cyv;
        if (mode == 3) return;
        if (S.hist && S.hist_row < S.hist_cap) {
            double* row = S.hist + (size_t)S.hist_row * (NV + 4);
            for (int k = 0; k < NV; k++) row[k] = res[k];
            row[NV] = cxp; row[NV + 1] = cxv; row[NV + 2] = cyp; row[NV + 3] = cyv;
        }
        sc->hist_row = S.hist_row + 1;
        // the residual-drop stop measures from the largest residual so far (a free-stream start has a first
        // density residual of round-off size; the start-up transient then raises it)
        double r00 = S.res0[0];
        if (!S.have_res0) {
            for (int k = 0; k < NV; k++) sc->res0[k] = res[k];
            sc->have_res0 = 1;
            r00 = res[0];
        } else {
            for (int k = 0; k < NV; k++)
                if (res[k] > S.res0[k]) sc->res0[k] = res[k];
            r00 = fmax(r00, res[0]);
        }
        sc->steps = S.steps + 1;
        if (S.iter == p.dt_local_n) sc->dt_local = 0;
        S.iter++;
        sc->iter = S.iter;
        if (bad) sc->status = 4; // CSU_ERR_NONFINITE
        if (p.tube) {
            S.t += S.dt * p.stages / 2.0;
            sc->t = S.t;
            if (S.stop_after) sc->done = 1;
        }
        if (p.conv_tol > 0 && res[0] <= p.conv_tol * r00) sc->done = 1;
        else if (p.iter_cap > 0 && S.iter >= p.iter_cap) sc->done = 2;
        for (int k = 0; k < MAX_SWEEPS; k++) sc->sweep_max[k] = 0ULL;
    }
    if (mode == 2 && !S.fresh) {
        sc->dtmin_bits = 0x7ff0000000000000ULL;
        return;
    }
    if (mode == 2) sc->fresh = 0;
    if (mode == 0 || mode == 2) {
        // solverCalcDt (solver.c:925-950) for the next iteration, from the minimum gathered above
        double dt = bitsd(S.dtmin_bits);
        dt *= cfl_at(p, S.iter);
        if (p.tube && S.t + dt > p.tmax) {
            dt = (p.tmax - S.t);
            sc->stop_after = 1;
        }
        sc->dt = dt;
    }
    sc->dtmin_bits = 0x7ff0000000000000ULL;
}

} // namespace csu
