// hp_kernels.cuh -- sm_100a kernels of the explicit residual-and-update step.
//
// Included once per precision variant with HP_NS (namespace) and HP_R (the
// arithmetic type of gradients, limiter, reconstruction, HLLC, sources and
// viscous fluxes) defined.  Primitive recovery through the stiffened-gas
// pressure-equilibrium quadratic, the RK state update and the dt / residual
// reductions are FP64 in every variant.
//
// Every kernel is cell-centric: one thread owns one cell, evaluates its own 4
// faces in local face order 1..4 and writes only that cell.  This keeps the
// reference's per-cell summation order (src/sr_hllcbatten.F90:77-555), so the
// parity variant (compiled with -fmad=false) reproduces the CPU reference
// bit for bit, and it needs no atomics.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <type_traits>

#include "hp_device.h"

namespace hp {
namespace HP_NS {

using R = HP_R;

// ---------------------------------------------------------------------------
// Fortran MIN/MAX as the reference's build evaluates them: a NaN argument is
// skipped unless it is the first (pinned by the shipped Velocity.dat).
template <class T> __device__ __forceinline__ T mn2(T a, T b) { return (b < a || a != a) ? b : a; }
template <class T> __device__ __forceinline__ T mx2(T a, T b) { return (b > a || a != a) ? b : a; }

// det() of src/mod_MatrixOps.F90:4-9
template <class T>
__device__ __forceinline__ T det3(T A11, T A21, T A31, T A12, T A22, T A32, T A13, T A23, T A33) {
    return A11 * (A22 * A33 - A23 * A32) - A21 * (A12 * A33 - A13 * A32) + A31 * (A12 * A23 - A13 * A22);
}
// fvenkat() of src/mod_MatrixOps.F90:12-18
template <class T>
__device__ __forceinline__ T fvenkat(T delp, T delm, T epssq) {
    return (((delp * delp + epssq) * delm + T(2) * delm * delm * delp) /
            (delp * delp + T(2) * delm * delm + delp * delm + epssq)) / delm;
}

template <class T> __device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

// Minimum resident 128-thread blocks per SM of the 4-lanes-per-cell kernels
// (sets their register cap: 65536 / (128 * minb)).
#ifndef HP_GRAD4_MINB
#define HP_GRAD4_MINB 4
#endif
#ifndef HP_FLUX4_MINB
#define HP_FLUX4_MINB 4
#endif
#ifndef HP_VISC4_MINB
#define HP_VISC4_MINB 3
#endif

// ---------------------------------------------------------------------------
// Division.  The parity path must return the IEEE round-to-nearest quotient
// of every division the reference performs.  Where several quotients share a
// divisor b, the fast form (F = 1) takes rb = RN(1/b) once and each a / b as
//     q0 = RN(a rb),  q1 = RN(q0 + RN(a - b q0) rb),  q2 = RN(q1 + (a - b q1) rb)
// with fused multiply-adds.  Markstein's theorem (rb within half an ulp of
// 1/b and q1 within one ulp of a/b make a - b q1 exact and q2 = RN(a/b),
// barring underflow and overflow) gives the IEEE quotient whenever |b| lies
// in [2^-100, 2^101) and |q2| in [2^-800, 2^801); a == 0 returns RN(a rb),
// the correctly signed zero.  Any other operand (out of range, Inf, NaN)
// sets `bad` instead, and the kernel whose warp saw it redoes its work with
// hardware division (F = 0), so every stored quotient is the IEEE one.  The
// fast form is straight-line FMA code that the compiler interleaves across
// independent divisions.
#ifndef HP_DIV_FAST
#define HP_DIV_FAST 0
#endif
#ifndef HP_S
#define HP_S double
#endif
// FP32-arithmetic variants with a face list: viscous fluxes evaluated once
// per face (1) instead of once from each side (0)
#ifndef HP_FACE_VISC
#define HP_FACE_VISC 1
#endif
// viscous fluxes of the cell-centric variants with eight lanes per cell (one
// phase each, k_visc8) instead of four (k_visc4)
// FP64 four-lane kernels: neighbour centroid differences from the set-up
// table m.dxn instead of gathered centroids
#ifndef HP_DXN_TABLE
#define HP_DXN_TABLE 1
#endif
#ifndef HP_VISC_SPLIT
#define HP_VISC_SPLIT 1
#endif
// kernels that take the fast form when HP_DIV_FAST is set: 1 gradients,
// 2 fluxes, 4 viscous fluxes, 8 JST smoothing
#ifndef HP_FAST_MASK
#define HP_FAST_MASK 15
#endif
#define HP_FAST(bit) (HP_DIV_FAST && (HP_FAST_MASK & (bit)) && sizeof(R) == 8)
template <int F>
__device__ __forceinline__ double mdiv(double a, double b, double rb, unsigned& bad) {
    if constexpr (F == 0) {
        (void)rb; (void)bad;
        return a / b;
    } else {
        const double q0 = a * rb;
        const double q1 = fma(fma(-b, q0, a), rb, q0);
        const double q2 = fma(fma(-b, q1, a), rb, q1);
        const unsigned eq = ((unsigned)__double2hiint(q2) >> 20) & 0x7ffu;
        const bool z = a == 0.0;
        bad |= (unsigned)(!z && eq - 223u > 1600u);
        return z ? q0 : q2;
    }
}
template <int F>
__device__ __forceinline__ double mrcp(double b, unsigned& bad) {
    if constexpr (F == 0) {
        (void)b; (void)bad;
        return 0.0;
    } else {
        const unsigned eb = ((unsigned)__double2hiint(b) >> 20) & 0x7ffu;
        bad |= (unsigned)(eb - 923u > 200u);
        return 1.0 / b;
    }
}
// mrcp with the reciprocal taken from a set-up table (rbt = RN(1/b)
// computed on the host): the same value and the same range flag, without
// the division
template <int F>
__device__ __forceinline__ double mrcp_tab(double b, double rbt, unsigned& bad) {
    if constexpr (F == 0) {
        (void)b; (void)rbt; (void)bad;
        return 0.0;
    } else {
        const unsigned eb = ((unsigned)__double2hiint(b) >> 20) & 0x7ffu;
        bad |= (unsigned)(eb - 923u > 200u);
        return rbt;
    }
}
template <int F> __device__ __forceinline__ float mrcp_tab(float b, float, unsigned& bad) {
    return mrcp<F>(b, bad);
}
// the mixed variant divides approximately
template <int F> __device__ __forceinline__ float mdiv(float a, float b, float rb, unsigned&) { return a * rb; }
template <int F> __device__ __forceinline__ float mrcp(float b, unsigned&) { return 1.0f / b; }

// One face record (FACE_REC values of R) of the face-based variants; the
// record of face t starts at FACE_REC * t, 16-byte aligned in FP32.  NC:
// through the read-only (non-coherent) data path, which a kernel may use
// only for data it does not write itself; the fused step, which writes the
// records in an earlier phase, reads them with plain loads.
template <bool NC = true>
__device__ __forceinline__ void load_frec(const float* p, float e[FACE_REC]) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a = NC ? __ldg(q) : q[0], b = NC ? __ldg(q + 1) : q[1], c = NC ? __ldg(q + 2) : q[2];
    e[0] = a.x; e[1] = a.y; e[2] = a.z; e[3] = a.w;
    e[4] = b.x; e[5] = b.y; e[6] = b.z; e[7] = b.w;
    e[8] = c.x; e[9] = c.y; e[10] = c.z; e[11] = c.w;
}
template <bool NC = true>
__device__ __forceinline__ void load_frec(const double* p, double e[FACE_REC]) {
#pragma unroll
    for (int k = 0; k < FACE_REC; k++) e[k] = NC ? __ldg(p + k) : p[k];
}
__device__ __forceinline__ void store_frec(float* p, const float e[FACE_REC]) {
    float4* q = reinterpret_cast<float4*>(p);
    q[0] = make_float4(e[0], e[1], e[2], e[3]);
    q[1] = make_float4(e[4], e[5], e[6], e[7]);
    q[2] = make_float4(e[8], e[9], e[10], e[11]);
}
__device__ __forceinline__ void store_frec(double* p, const double e[FACE_REC]) {
#pragma unroll
    for (int k = 0; k < FACE_REC; k++) p[k] = e[k];
}

// Exact division at sites that are not on the fast path.
__device__ __forceinline__ double div_rn(double a, double b, double) { return a / b; }
__device__ __forceinline__ float div_rn(float a, float b, float rb) { return a * rb; }
__device__ __forceinline__ double rcp(double) { return 0.0; }
__device__ __forceinline__ float rcp(float b) { return 1.0f / b; }

// Value of lane q of this thread's group of four consecutive lanes.
template <class T>
__device__ __forceinline__ T qshfl(T v, int q) {
    return __shfl_sync(0xffffffffu, v, (int)((threadIdx.x & 31) & ~3u) + q);
}

#define COL(ptr, k) ((ptr) + (size_t)(k) * (size_t)m.ld)

// case of element i (0 for a single-case handle)
__device__ __forceinline__ int case_of(const DevMesh& m, int i) { return m.cid ? ldg(m.cid + i) : 0; }

// ---------------------------------------------------------------------------
// Primitive recovery, src/sr_primitive.F90:23-161 (== the element loop of
// src/sr_primitiveplusbc.F90:36-172 without ag/ap).  c[] is renormalised.
// S is the arithmetic of the state path (EOS recovery, RK update, JST, dt):
// double in every variant except the all-FP32 one.
using S = HP_S;

struct PrimV {
    S ug, vg, wg, tg, pg, pp, phig, phip, up, vp, wp, tp, rog, rop;
};

__device__ __forceinline__ void blend_phases(const DevParams& P, S& phig, S& phip, S& ug, S& vg, S& wg, S& tg,
                                             S& pg, S& up, S& vp, S& wp, S& tp, S& pp) {
    const S emin = (S)P.emin, emax = (S)P.emax;
    if (phig < emin) {
        phig = emin; phip = S(1.0) - phig;
        ug = up; vg = vp; wg = wp; tg = tp; pg = pp;
    }
    if (phip < emin) {
        phip = emin; phig = S(1.0) - phip;
        up = ug; vp = vg; wp = wg; tp = tg; pp = pg;
    }
    if (phig >= emin && phig <= emax) {
        S psig = div_rn(phig - emin, emax - emin, (S)P.r_emm);
        S f = -(psig * psig * (S(2.0) * psig - S(3.0)));
        ug = f * ug + (S(1.0) - f) * up;
        vg = f * vg + (S(1.0) - f) * vp;
        wg = f * wg + (S(1.0) - f) * wp;
        tg = f * tg + (S(1.0) - f) * tp;
        pg = f * pg + (S(1.0) - f) * pp;
    }
    if (phip >= emin && phip <= emax) {
        S psig = div_rn(phip - emin, emax - emin, (S)P.r_emm);
        S f = -(psig * psig * (S(2.0) * psig - S(3.0)));
        up = f * up + (S(1.0) - f) * ug;
        vp = f * vp + (S(1.0) - f) * vg;
        wp = f * wp + (S(1.0) - f) * wg;
        tp = f * tp + (S(1.0) - f) * tg;
        pp = f * pp + (S(1.0) - f) * pg;
    }
}

// qm: the dispersed masses cn(11), cn(15), cn(19) of the five-phase model
// (src/sr_primitive.F90:56-80), or null for the two-phase model
__device__ __forceinline__ void prim_full(double cd[10], PrimV& q, const DevParams& P,
                                          const double* qm = nullptr) {
    S c[10];
#pragma unroll
    for (int k = 0; k < 10; k++) c[k] = (S)cd[k];
    const S gamag = (S)P.gamag, gamap = (S)P.gamap, pinf = (S)P.pinf, fsd = (S)P.fsd;
    const S rrg = (S)P.rrg, cpp = (S)P.cpp;
    const S r0 = rcp(c[0]), r5 = rcp(c[5]);
    q.ug = div_rn(c[1], c[0], r0); q.vg = div_rn(c[2], c[0], r0); q.wg = div_rn(c[3], c[0], r0);
    q.up = div_rn(c[6], c[5], r5); q.vp = div_rn(c[7], c[5], r5); q.wp = div_rn(c[8], c[5], r5);
    S eg = div_rn(c[4], c[0], r0) - S(0.5) * (q.ug * q.ug + q.vg * q.vg + q.wg * q.wg);
    S ep = div_rn(c[9], c[5], r5) - S(0.5) * (q.up * q.up + q.vp * q.vp + q.wp * q.wp);
    if (qm) {
        // the dispersed phases take their share of the volume out of the
        // pressure-equilibrium quadratic; densities from the energies
        const S emin = (S)P.emin;
        const S phq = mn2(mx2((S)qm[0] / (S)P.rhod[0], emin), S(1.0) - emin);
        const S phr = mn2(mx2((S)qm[1] / (S)P.rhod[1], emin), S(1.0) - emin);
        const S phs = mn2(mx2((S)qm[2] / (S)P.rhod[2], emin), S(1.0) - emin);
        const S aaa = mn2(mx2(S(1.0) - phq - phr - phs, emin), S(1.0) - emin);
        S bbb = (aaa * pinf * gamap) - (c[0] * (gamag - S(1.0)) * eg) - (c[5] * (gamap - S(1.0)) * ep);
        S ccc = (c[0] * (gamag - S(1.0)) * eg * (gamap * pinf));
        q.pg = (-bbb + sqrt(bbb * bbb + S(4.0) * aaa * ccc)) / (S(2.0) * aaa);
        q.pp = q.pg + fsd;
        q.rog = q.pg / ((gamag - S(1.0)) * eg);
        q.rop = (q.pp + pinf * gamap) / ((gamap - S(1.0)) * ep);
        q.tg = q.pg / (q.rog * rrg);
        q.tp = ((q.pp + pinf) * gamap) / ((gamap - S(1.0)) * q.rop * cpp);
        q.phig = mn2(mx2(c[0] / q.rog, emin), S(1.0) - emin);
        q.phip = mn2(mx2(c[5] / q.rop, emin), S(1.0) - emin);
    } else {
        S bbb = (fsd + pinf * gamap) - (c[0] * (gamag - S(1.0)) * eg) - (c[5] * (gamap - S(1.0)) * ep);
        S ccc = c[0] * (gamag - S(1.0)) * eg * (fsd + pinf * gamap);
        q.pg = (-bbb + sqrt(bbb * bbb + S(4.0) * ccc)) * S(0.5);
        q.pp = q.pg + fsd;
        q.phig = (c[0] * (gamag - S(1.0)) * eg) / q.pg;
        q.phip = S(1.0) - q.phig;
        q.rog = c[0] / q.phig;
        q.rop = c[5] / q.phip;
        q.tg = q.pg / (q.rog * rrg);
        q.tp = ((q.pp + pinf) * gamap) / ((gamap - S(1.0)) * q.rop * cpp);
    }
    blend_phases(P, q.phig, q.phip, q.ug, q.vg, q.wg, q.tg, q.pg, q.up, q.vp, q.wp, q.tp, q.pp);
    q.rog = q.pg / (rrg * q.tg);
    q.rop = (q.pp + pinf) * gamap / ((gamap - S(1.0)) * cpp * q.tp);
    S eg2 = q.pg / ((gamag - S(1.0)) * q.rog);
    S ep2 = (q.pp + gamap * pinf) / ((gamap - S(1.0)) * q.rop);
    S egt = eg2 + S(0.5) * (q.ug * q.ug + q.vg * q.vg + q.wg * q.wg);
    S ept = ep2 + S(0.5) * (q.up * q.up + q.vp * q.vp + q.wp * q.wp);
    cd[0] = q.phig * q.rog;
    cd[1] = q.phig * q.rog * q.ug;
    cd[2] = q.phig * q.rog * q.vg;
    cd[3] = q.phig * q.rog * q.wg;
    cd[4] = q.phig * q.rog * egt;
    cd[5] = q.phip * q.rop;
    cd[6] = q.phip * q.rop * q.up;
    cd[7] = q.phip * q.rop * q.vp;
    cd[8] = q.phip * q.rop * q.wp;
    cd[9] = q.phip * q.rop * ept;
}

template <class T>
__device__ __forceinline__ void store_prims(const DevMesh& m, T* pr, int i, const PrimV& q) {
    COL(pr, P_UG)[i] = (T)q.ug; COL(pr, P_VG)[i] = (T)q.vg; COL(pr, P_WG)[i] = (T)q.wg;
    COL(pr, P_TG)[i] = (T)q.tg; COL(pr, P_PG)[i] = (T)q.pg; COL(pr, P_PP)[i] = (T)q.pp;
    COL(pr, P_PHIG)[i] = (T)q.phig; COL(pr, P_PHIP)[i] = (T)q.phip;
    COL(pr, P_UP)[i] = (T)q.up; COL(pr, P_VP)[i] = (T)q.vp; COL(pr, P_WP)[i] = (T)q.wp;
    COL(pr, P_TP)[i] = (T)q.tp; COL(pr, P_ROG)[i] = (T)q.rog; COL(pr, P_ROP)[i] = (T)q.rop;
}

// Block-wide min / max of 64-bit keys, then one atomic per block.
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

enum { PM_STAGE = 0, PM_START = 1, PM_END = 2 };

// Element primitive pass.  PM_START adds the dt contribution of
// src/main.F90:529-546; PM_END adds the max-norm residual of :605-611, the
// cu = cn copy of :619-625 and |u_g(1)| of :641.
template <int MODE>
__device__ __forceinline__ void k_prim_body(DevMesh m, DevState<R> s, DevParams P, int bid) {
    __shared__ unsigned long long red[4][16];
    int i = bid * blockDim.x + threadIdx.x;
    unsigned long long kmin = ~0ull, kd[4] = {0, 0, 0, 0}, nanc = 0;
    if (i < m.neles) {
        double c[10], u[10];
#pragma unroll
        for (int k = 0; k < 10; k++) c[k] = COL(s.cn, k)[i];
        // cu is read before any store of this thread: the compiler cannot
        // prove cn, cu and the primitive columns disjoint, so a load after a
        // store would wait for it
        if (MODE == PM_END) {
#pragma unroll
            for (int k = 0; k < 10; k++) u[k] = COL(s.cu, k)[i];
        }
        PrimV q;
        double qm[3];
        if (P.five_phase) {
            qm[0] = COL(s.cn, 10)[i]; qm[1] = COL(s.cn, 14)[i]; qm[2] = COL(s.cn, 18)[i];
        }
        prim_full(c, q, P, P.five_phase ? qm : nullptr);
#pragma unroll
        for (int k = 0; k < 10; k++) COL(s.cn, k)[i] = c[k];
        store_prims(m, s.pr, i, q);
        if constexpr (sizeof(R) != sizeof(double)) store_prims(m, s.prr, i, q);
        if (MODE == PM_START) {
            S ag = sqrt(((S)P.gamag * q.pg) / q.rog);
            S ap = sqrt(((S)P.gamap * (q.pp + (S)P.pinf)) / q.rop);
            S qg = sqrt(q.ug * q.ug + q.vg * q.vg + q.wg * q.wg);
            S qp = sqrt(q.up * q.up + q.vp * q.vp + q.wp * q.wp);
            S x = (S)ldg(m.dl + i) / (mx2(ag, ap) + mx2(qg, qp));
            if (x == x) kmin = (unsigned long long)__double_as_longlong((double)x);
        }
        if (MODE == PM_END) {
            bool bad = false;
#pragma unroll
            for (int k = 0; k < 10; k++) {
                if (k < 4) {
                    double d = fabs(c[k] - u[k]);
                    if (d == d) kd[k] = (unsigned long long)__double_as_longlong(d);
                }
                bad |= (c[k] != c[k]);
                COL(s.cu, k)[i] = c[k];
            }
            if (P.five_phase) {   // cu = cn over all 22 variables (src/main.F90:619-625)
                for (int k = 10; k < 22; k++) {
                    const double v = COL(s.cn, k)[i];
                    bad |= (v != v);
                    COL(s.cu, k)[i] = v;
                }
            }
            // halo cells are counted by the part that owns them
            nanc = (bad && ldg(m.iblank + i) < HP_IBLANK_HALO1) ? 1 : 0;
            DevScalars& sc = s.s[case_of(m, i)];
            if (i == sc.cell1) sc.velmag = sqrt(q.ug * q.ug + q.vg * q.vg + q.wg * q.wg);
        }
    }
    if (MODE == PM_STAGE) return;
    // a block whose cells belong to two cases of a batch reduces per thread
    // (block-uniform branch: cases occupy contiguous element ranges)
    const int b0 = bid * blockDim.x;
    const int c0 = case_of(m, b0), c1 = case_of(m, min(b0 + (int)blockDim.x, m.neles) - 1);
    if (c0 != c1) {
        if (i < m.neles) {
            DevScalars& sc = s.s[case_of(m, i)];
            if (MODE == PM_START) {
                if (kmin != ~0ull) atomicMin(&sc.dtmin_bits, kmin);
            } else {
                for (int k = 0; k < 4; k++)
                    if (kd[k]) atomicMax(&sc.diff_bits[k], kd[k]);
                if (nanc) atomicAdd(&sc.nan_count, nanc);
            }
        }
        return;
    }
    DevScalars* const S0 = s.s + c0;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (MODE == PM_START) {
        kmin = warp_min_u64(kmin);
        if (lane == 0) red[0][wid] = kmin;
        __syncthreads();
        if (wid == 0) {
            unsigned long long v = lane < (int)(blockDim.x >> 5) ? red[0][lane] : ~0ull;
            v = warp_min_u64(v);
            if (lane == 0 && v != ~0ull) atomicMin(&S0->dtmin_bits, v);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) kd[k] = warp_max_u64(kd[k]);
        for (int o = 16; o > 0; o >>= 1) nanc += __shfl_xor_sync(0xffffffffu, nanc, o);
        if (lane == 0) {
            for (int k = 0; k < 4; k++) red[k][wid] = kd[k];
        }
        __shared__ unsigned long long nred[16];
        if (lane == 0) nred[wid] = nanc;
        __syncthreads();
        if (wid == 0) {
            int nw = blockDim.x >> 5;
            for (int k = 0; k < 4; k++) {
                unsigned long long v = lane < nw ? red[k][lane] : 0ull;
                v = warp_max_u64(v);
                if (lane == 0 && v) atomicMax(&S0->diff_bits[k], v);
            }
            unsigned long long c = lane < nw ? nred[lane] : 0ull;
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0 && c) atomicAdd(&S0->nan_count, c);
        }
    }
}
template <int MODE>
__global__ void __launch_bounds__(512) k_prim(DevMesh m, DevState<R> s, DevParams P) {
    k_prim_body<MODE>(m, s, P, blockIdx.x);
}

// dt = cfl * dtmin, time += dt (src/main.F90:521-556); one thread per case.
__device__ __forceinline__ void step_begin_case(DevScalars* sc, const DevParams& P, unsigned long long bits) {
    double dtmin = __longlong_as_double((long long)bits);
    sc->dt = dtmin * P.cfl;
    sc->time = sc->time + sc->dt;
    sc->total = sc->total + 1;
    sc->dtmin_bits = (unsigned long long)__double_as_longlong(1.0e8);
}

// One thread per case.  coupled: the cases are the parts of one mesh and all
// take the minimum over all of them (the positive dt contributions order as
// their bit patterns); launched as one block, which reads every case before
// any is reset.
__global__ void k_step_begin(DevState<R> s, DevParams P, int ncase, int coupled) {
    if (coupled) {
        unsigned long long bits = ~0ull;
        for (int k = 0; k < ncase; k++) bits = min(bits, s.s[k].dtmin_bits);
        __syncthreads();
        for (int c = threadIdx.x; c < ncase; c += blockDim.x) step_begin_case(s.s + c, P, bits);
        return;
    }
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < ncase) step_begin_case(s.s + c, P, s.s[c].dtmin_bits);
}

// per-step diagnostics and reset of the residual accumulators; one thread
// per case (diag rows of case c start at c * max_diag).
__device__ __forceinline__ void k_step_end_body(DevState<R> s, int ncase, int bid) {
    const int c = bid * blockDim.x + threadIdx.x;
    if (c >= ncase) return;
    DevScalars* sc = s.s + c;
    int k = sc->step_in_call;
    if (k < s.max_diag) {
        double* d = s.diag + 8 * ((size_t)c * s.max_diag + k);
        d[0] = sc->time; d[1] = sc->dt; d[2] = sc->velmag;
        for (int j = 0; j < 4; j++) d[3 + j] = __longlong_as_double((long long)sc->diff_bits[j]);
        d[7] = (double)sc->nan_count;
    }
    sc->step_in_call = k + 1;
    for (int j = 0; j < 4; j++) sc->diff_bits[j] = 0ull;
    sc->nan_count = 0ull;
}
__global__ void k_step_end(DevState<R> s, int ncase) {
    k_step_end_body(s, ncase, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Ghost states per boundary type, src/sr_primitiveplusbc.F90:198-592
// (VISC = false) and src/sr_viscousgp.F90:71-446 (VISC = true).  Types 6
// (isothermal no-slip wall) and 7 (far field) are additions of this build.
// Operates on one ghost-list entry; reads the parent's primitives and the
// ghost's previous primitives.
template <bool VISC>
__device__ __forceinline__ void bc_one(const DevMesh& m, double* pr, double* egt, const DevParams& P,
                                       int gidx, double dt, int total) {
    const int np = m.g_par[gidx], ng = m.g_id[gidx], nt = m.g_type[gidx];
    double* ug = COL(pr, P_UG); double* vg = COL(pr, P_VG); double* wg = COL(pr, P_WG);
    double* tg = COL(pr, P_TG); double* pg = COL(pr, P_PG); double* pp = COL(pr, P_PP);
    double* phig = COL(pr, P_PHIG); double* phip = COL(pr, P_PHIP);
    double* up = COL(pr, P_UP); double* vp = COL(pr, P_VP); double* wp = COL(pr, P_WP);
    double* tp = COL(pr, P_TP); double* rog = COL(pr, P_ROG); double* rop = COL(pr, P_ROP);
    const double rrg = P.rrg, gamag = P.gamag, gamap = P.gamap, pinf = P.pinf, cpp = P.cpp;
    if (nt == 2) {
        phip[ng] = P.phipzero;
        // five-phase: the dispersed fractions at the inflow are epslnmin
        // (src/sr_primitiveplusbc.F90:210-216, src/sr_viscousgp.F90:83-88)
        if (P.five_phase) phig[ng] = 1.0 - phip[ng] - P.emin - P.emin - P.emin;
        else phig[ng] = 1.0 - phip[ng];
        ug[ng] = P.ugmin; vg[ng] = P.vgmin; wg[ng] = P.wgmin;
        tg[ng] = P.tgmin;
        pg[ng] = pg[np];
        rog[ng] = pg[ng] / (rrg * tg[ng]);
        up[ng] = 0.99 * P.ugmin; vp[ng] = 0.99 * P.vgmin; wp[ng] = 0.99 * P.wgmin;
        tp[ng] = P.tgmin;
        pp[ng] = pp[np];
        rop[ng] = gamap * (pg[ng] + pinf) / ((gamap - 1.0) * cpp * tp[ng]);
    } else if (nt == 3) {
        phig[ng] = phig[np];
        phip[ng] = phip[np];
        double dd = m.dd[np];
        double wT = ug[np];
        double wU = ug[np] + sqrt(gamag * pg[np] / rog[np]);
        double alphaT = wT * dt / dd, alphaU = wU * dt / dd;
        double fracT = 1 / (1 + alphaT), fracU = 1 / (1 + alphaU);
        if (total == 1) {
            ug[ng] = ug[np]; vg[ng] = vg[np]; wg[ng] = wg[np]; tg[ng] = tg[np]; pg[ng] = P.pmin;
        }
        if (ug[np] > ug[ng]) {
            ug[ng] = ug[ng] * fracU + (1 - fracU) * (2.0 * ug[np] - ug[ng]);
            vg[ng] = vg[ng] * fracT + (1 - fracT) * (2.0 * vg[np] - vg[ng]);
            wg[ng] = wg[ng] * fracT + (1 - fracT) * (2.0 * wg[np] - wg[ng]);
            tg[ng] = tg[ng] * fracT + (1 - fracT) * (2.0 * tg[np] - tg[ng]);
        } else {
            ug[ng] = ug[np]; vg[ng] = vg[np]; wg[ng] = wg[np]; tg[ng] = tg[np];
        }
        pg[ng] = P.pmin;
        rog[ng] = pg[ng] / (rrg * tg[ng]);
        vp[ng] = vp[np]; up[ng] = up[np]; wp[ng] = wp[np];
        pp[ng] = P.pmin;
        tp[ng] = tp[np];
        rop[ng] = gamap * (pp[ng] + pinf) / ((gamap - 1.0) * cpp * tp[ng]);
    } else if (nt == 5) {
        phig[ng] = phig[np];
        ug[ng] = -ug[np]; vg[ng] = -vg[np]; wg[ng] = -wg[np];
        tg[ng] = tg[np];
        phip[ng] = phip[np];
        up[ng] = -up[np]; vp[ng] = -vp[np]; wp[ng] = -wp[np];
        tp[ng] = tp[np];
        pg[ng] = pg[np]; pp[ng] = pp[np];
        rog[ng] = pg[ng] / (rrg * tg[ng]);
        rop[ng] = gamap * (pp[ng] + pinf) / ((gamap - 1.0) * cpp * tp[ng]);
    } else if (nt == 51 || nt == 53) {
        const bool ylat = (nt == 51);
        double* vn = ylat ? vg : wg;
        double* t2 = ylat ? wg : vg;
        double dd = m.dd[np];
        double wT = vn[np];
        double alphaT = wT * dt / dd;
        double fracT = 1 / (1 + alphaT);
        if (vn[np] > vn[ng]) {
            if (VISC && !ylat) vn[ng] = -vn[ng];   // src/sr_viscousgp.F90:408
            else vn[ng] = -vn[np];
            ug[ng] = ug[ng] * fracT + (1 - fracT) * (2.0 * ug[np] - ug[ng]);
            t2[ng] = t2[ng] * fracT + (1 - fracT) * (2.0 * t2[np] - t2[ng]);
            tg[ng] = tg[ng] * fracT + (1 - fracT) * (2.0 * tg[np] - tg[ng]);
        } else {
            ug[ng] = ug[np]; vn[ng] = -vn[np]; t2[ng] = t2[np]; tg[ng] = tg[np];
        }
        pg[ng] = pg[np];
        phig[ng] = phig[np];
        phip[ng] = phip[np];
        up[ng] = up[np]; vp[ng] = vp[np]; wp[ng] = wp[np];
        if (ylat) vp[ng] = -vp[np]; else wp[ng] = -wp[np];
        tp[ng] = tp[np];
        pp[ng] = pp[np];
        rog[ng] = pg[ng] / (rrg * tg[ng]);
        rop[ng] = gamap * (pp[ng] + pinf) / ((gamap - 1.0) * cpp * tp[ng]);
    } else if (nt == 6) {
        phig[ng] = phig[np]; phip[ng] = phip[np];
        ug[ng] = -ug[np]; vg[ng] = -vg[np]; wg[ng] = -wg[np];
        up[ng] = -up[np]; vp[ng] = -vp[np]; wp[ng] = -wp[np];
        tg[ng] = 2.0 * P.twall - tg[np];
        tp[ng] = 2.0 * P.twall - tp[np];
        pg[ng] = pg[np]; pp[ng] = pp[np];
        rog[ng] = pg[ng] / (rrg * tg[ng]);
        rop[ng] = gamap * (pp[ng] + pinf) / ((gamap - 1.0) * cpp * tp[ng]);
    } else if (nt == 7) {
        phip[ng] = P.phipzero; phig[ng] = 1.0 - phip[ng];
        ug[ng] = P.ugmin; vg[ng] = P.vgmin; wg[ng] = P.wgmin;
        up[ng] = P.upmin; vp[ng] = P.vpmin; wp[ng] = P.wpmin;
        tg[ng] = P.tgmin; tp[ng] = P.tpmin;
        pg[ng] = P.pmin; pp[ng] = P.pmin + P.fsd;
        rog[ng] = pg[ng] / (rrg * tg[ng]);
        rop[ng] = gamap * (pp[ng] + pinf) / ((gamap - 1.0) * cpp * tp[ng]);
    }
    if (!VISC && egt != nullptr && (nt == 2 || nt == 3 || nt == 5 || nt == 51 || nt == 53 || nt == 6 || nt == 7)) {
        // egtotal / eptotal of the ghost as the BC loop that wrote it last
        // defines them (src/sr_primitiveplusbc.F90:255-258 for type 2,
        // :342-345 and siblings for the others)
        double eg, ep;
        if (nt == 2) {
            eg = pg[ng] / (rog[ng] * (gamag - 1.0));
            ep = (pp[ng] + gamap * pinf) / (rop[ng] * (gamap - 1.0));
        } else {
            eg = rrg * tg[ng] / (gamag - 1.0);
            ep = cpp * tp[ng] / gamap + pinf / rop[ng];
        }
        egt[ng] = eg + 0.5 * (ug[ng] * ug[ng] + vg[ng] * vg[ng] + wg[ng] * wg[ng]);
        egt[m.ld + ng] = ep + 0.5 * (up[ng] * up[ng] + vp[ng] * vp[ng] + wp[ng] * wp[ng]);
    }
}

// ghost cn, src/sr_primitiveplusbc.F90:602-631 (energies as the BC loops
// define them; only observable when ghost ids alias element ids)
__device__ __forceinline__ void ghost_cn_one(const DevMesh& m, double* pr, double* cn,
                                             const double* egtp, int gidx) {
    const int ng = m.g_id[gidx];
    double ug = COL(pr, P_UG)[ng], vg = COL(pr, P_VG)[ng], wg = COL(pr, P_WG)[ng];
    double up = COL(pr, P_UP)[ng], vp = COL(pr, P_VP)[ng], wp = COL(pr, P_WP)[ng];
    double phig = COL(pr, P_PHIG)[ng], phip = COL(pr, P_PHIP)[ng];
    double rog = COL(pr, P_ROG)[ng], rop = COL(pr, P_ROP)[ng];
    double egt = egtp[ng], ept = egtp[m.ld + ng];
    COL(cn, 0)[ng] = phig * rog; COL(cn, 1)[ng] = phig * rog * ug;
    COL(cn, 2)[ng] = phig * rog * vg; COL(cn, 3)[ng] = phig * rog * wg;
    COL(cn, 4)[ng] = phig * rog * egt; COL(cn, 5)[ng] = phip * rop;
    COL(cn, 6)[ng] = phip * rop * up; COL(cn, 7)[ng] = phip * rop * vp;
    COL(cn, 8)[ng] = phip * rop * wp; COL(cn, 9)[ng] = phip * rop * ept;
}

// Parallel ghost fill: valid when every ghost id is its own slot and every
// parent is an element (no aliasing), so ghost entries are independent.
template <bool VISC>
__device__ __forceinline__ void k_bc_body(DevMesh m, DevState<R> s, DevParams P, int bid) {
    int g = bid * blockDim.x + threadIdx.x;
    if (g >= m.nghosts) return;
    const DevScalars& sc = s.s[case_of(m, m.g_par[g])];
    bc_one<VISC>(m, s.pr, nullptr, P, g, sc.dt, sc.total);
    if constexpr (sizeof(R) != sizeof(double)) {
        const int ng = m.g_id[g];
#pragma unroll
        for (int k = 0; k < NPR; k++) COL(s.prr, k)[ng] = (R)COL(s.pr, k)[ng];
    }
}
template <bool VISC>
__global__ void __launch_bounds__(512) k_bc(DevMesh m, DevState<R> s, DevParams P) {
    k_bc_body<VISC>(m, s, P, blockIdx.x);
}

// Sequential ghost fill in the reference's exact order (type lists 2, 3, 5,
// 51, 53, then ghost cn for every ghost) for meshes whose ghost ids alias
// element ids or each other (e.g. merged overset meshes).  One thread.
template <bool VISC>
__global__ void k_bc_serial(DevMesh m, DevState<R> s, DevParams P) {
    const int order[7] = {2, 3, 5, 51, 53, 6, 7};
    double dt = s.s->dt;
    int total = s.s->total;
    for (int t = 0; t < 7; t++)
        for (int g = 0; g < m.nghosts; g++)
            if (m.g_type[g] == order[t]) bc_one<VISC>(m, s.pr, VISC ? nullptr : s.egt, P, g, dt, total);
    if (!VISC)
        for (int g = 0; g < m.nghosts; g++) ghost_cn_one(m, s.pr, s.cn, s.egt, g);
}

// src/sr_smooth.F90:19-41 and :164-187 ghost copies (aliased meshes only;
// otherwise the smoothing kernels read the parent through m.snb).
__global__ void k_smooth_copy_serial(DevMesh m, DevState<R> s, int which) {
    for (int g = 0; g < m.nghosts; g++) {
        int ng = m.g_id[g], np = m.g_par[g];
        if (which == 0) {
            COL(s.pr, P_PG)[ng] = COL(s.pr, P_PG)[np];
            COL(s.pr, P_PP)[ng] = COL(s.pr, P_PP)[np];
            for (int k = 0; k < 10; k++) COL(s.cn, k)[ng] = COL(s.cn, k)[np];
        } else {
            for (int k = 0; k < 10; k++) COL(s.d2q, k)[ng] = COL(s.d2q, k)[np];
            COL(s.anu, 0)[ng] = COL(s.anu, 0)[np];
            COL(s.anu, 1)[ng] = COL(s.anu, 1)[np];
        }
    }
}

// phi(ghost) = phi(parent), src/sr_VK.F90:299-301 (aliased meshes only).
__global__ void k_phi_copy_serial(DevMesh m, DevState<R> s) {
    for (int g = 0; g < m.nghosts; g++) s.phi[m.g_id[g]] = s.phi[m.g_par[g]];
}

// ---------------------------------------------------------------------------
// JST dissipation, src/sr_smooth.F90:52-154: switches anu and Laplacian d2q.
//
// The standalone k_smooth1 (HP_JST_SETS) runs two threads per cell: the
// first half of a block takes variables 1-5 and the gas-pressure switch of
// its cells, the second half variables 6-10 and the liquid-pressure switch,
// so each warp still reads one column for 32 consecutive cells and every
// thread has half the neighbour gathers in flight.  The values are those of
// the one-thread form (the fused step's).  (The same split of k_smooth2
// measured 16% slower: each thread repeats its volume gathers and
// divisions.)
#ifndef HP_JST_SETS
#define HP_JST_SETS 1
#endif
// set 0: variables 1-5, anu(:,1); set 1: variables 6-10, anu(:,2)
__device__ __forceinline__ void smooth1_set(const DevMesh& m, const DevState<R>& s, int i, int set) {
    const int a = ldg(COL(m.snb, 0) + i), b = ldg(COL(m.snb, 1) + i);
    const int c = ldg(COL(m.snb, 2) + i), d = ldg(COL(m.snb, 3) + i);
    const double* pq = COL(s.pr, set == 0 ? P_PG : P_PP);
    const S e6 = (S)(double)1.0e-6f;
    // switch sums of the set's first and last variable (1 and 5, or 6 and
    // 10) and the Laplacian of its five variables
    S swn[2], swd[2], lap[5];
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const double* col = COL(s.cn, 5 * set + k);
        const S v0 = (S)col[i], v1 = (S)col[a], v2 = (S)col[b], v3 = (S)col[c], v4 = (S)col[d];
        if (k == 0 || k == 4) {
            swn[k >> 2] = fabs(v1 - v0) + fabs(v2 - v0) + fabs(v3 - v0) + fabs(v4 - v0);
            swd[k >> 2] = fabs(v1 + v0) + fabs(v2 + v0) + fabs(v3 + v0) + fabs(v4 + v0);
        }
        lap[k] = v1 - v0 + v2 - v0 + v3 - v0 + v4 - v0;
    }
    const S qi = (S)pq[i], qa = (S)pq[a], qb = (S)pq[b], qc = (S)pq[c], qd = (S)pq[d];
    const S anun = fabs(qa - qi) + fabs(qb - qi) + fabs(qc - qi) + fabs(qd - qi);
    const S anud = fabs(qa + qi) + fabs(qb + qi) + fabs(qc + qi) + fabs(qd + qi);
    S anu;
    if (set == 0) {   // pressure, then variable 5, then variable 1
        anu = anun / anud + swn[1] / (swd[1] + e6);
        anu = anu + swn[0] / (swd[0] + e6);
    } else {          // pressure, then variable 6, then variable 10
        anu = anun / anud + swn[0] / (swd[0] + e6);
        anu = anu + swn[1] / (swd[1] + e6);
    }
#pragma unroll
    for (int k = 0; k < 5; k++) COL(s.d2q, 5 * set + k)[i] = lap[k];
    COL(s.anu, set)[i] = anu;
}
__device__ __forceinline__ void k_smooth1_body(DevMesh m, DevState<R> s, int bid) {
    int i = bid * blockDim.x + threadIdx.x;
    if (i >= m.neles) return;
    const int a = ldg(COL(m.snb, 0) + i), b = ldg(COL(m.snb, 1) + i);
    const int c = ldg(COL(m.snb, 2) + i), d = ldg(COL(m.snb, 3) + i);
    const double* pg = COL(s.pr, P_PG);
    const double* pp = COL(s.pr, P_PP);
    const S e6 = (S)(double)1.0e-6f;
    // the switch sums of variables 1, 5, 6, 10 (sw[0..3]) and the Laplacian
    // d2q of every variable, one variable at a time
    S swn[4], swd[4], lap[10];
#pragma unroll
    for (int k = 0; k < 10; k++) {
        const double* col = COL(s.cn, k);
        const S v0 = (S)col[i], v1 = (S)col[a], v2 = (S)col[b], v3 = (S)col[c], v4 = (S)col[d];
        const int slot = k == 0 ? 0 : k == 4 ? 1 : k == 5 ? 2 : k == 9 ? 3 : -1;
        if (slot >= 0) {
            swn[slot] = fabs(v1 - v0) + fabs(v2 - v0) + fabs(v3 - v0) + fabs(v4 - v0);
            swd[slot] = fabs(v1 + v0) + fabs(v2 + v0) + fabs(v3 + v0) + fabs(v4 + v0);
        }
        lap[k] = v1 - v0 + v2 - v0 + v3 - v0 + v4 - v0;
    }
    const S pgi = (S)pg[i], pga = (S)pg[a], pgb = (S)pg[b], pgc = (S)pg[c], pgd = (S)pg[d];
    S anun = fabs(pga - pgi) + fabs(pgb - pgi) + fabs(pgc - pgi) + fabs(pgd - pgi);
    S anud = fabs(pga + pgi) + fabs(pgb + pgi) + fabs(pgc + pgi) + fabs(pgd + pgi);
    S anupg = anun / anud;
    S anu1 = anupg + swn[1] / (swd[1] + e6);
    anu1 = anu1 + swn[0] / (swd[0] + e6);
    const S ppi = (S)pp[i], ppa = (S)pp[a], ppb = (S)pp[b], ppc = (S)pp[c], ppd = (S)pp[d];
    anun = fabs(ppa - ppi) + fabs(ppb - ppi) + fabs(ppc - ppi) + fabs(ppd - ppi);
    anud = fabs(ppa + ppi) + fabs(ppb + ppi) + fabs(ppc + ppi) + fabs(ppd + ppi);
    S anupp = anun / anud;
    S anu2 = anupp + swn[2] / (swd[2] + e6);
    anu2 = anu2 + swn[3] / (swd[3] + e6);
    // all stores after all loads (the output columns may alias the inputs
    // as far as the compiler can tell)
#pragma unroll
    for (int k = 0; k < 10; k++) COL(s.d2q, k)[i] = lap[k];
    COL(s.anu, 0)[i] = anu1;
    COL(s.anu, 1)[i] = anu2;
}
__global__ void __launch_bounds__(512) k_smooth1(DevMesh m, DevState<R> s) {
#if HP_JST_SETS
    const int half = (int)blockDim.x >> 1, set = (int)threadIdx.x >= half;
    const int i = blockIdx.x * half + ((int)threadIdx.x - set * half);
    if (i < m.neles) smooth1_set(m, s, i, set);
#else
    k_smooth1_body(m, s, blockIdx.x);
#endif
}

// src/sr_smooth.F90:200-374: blended 2nd/4th difference d24.  F selects the
// division form (see mdiv); returns the fast form's out-of-range flag.
template <int F>
__device__ __forceinline__ unsigned smooth2_body(const DevMesh& m, const DevState<R>& s, const DevParams& P, int i) {
    unsigned bad = 0;
    const S dt = (S)s.s[case_of(m, i)].dt;
    const S rdt = mrcp<F>(dt, bad);
    int nb[4];
#pragma unroll
    for (int f = 0; f < 4; f++) nb[f] = ldg(COL(m.snb, f) + i);
    const S vi = mdiv<F>((S)ldg(m.vol + i), dt, rdt, bad);
    S d24nc[4], out[10];
#pragma unroll
    for (int f = 0; f < 4; f++) d24nc[f] = S(0.5) * (vi + mdiv<F>((S)ldg(m.vol + nb[f]), dt, rdt, bad));
#pragma unroll
    for (int set = 0; set < 2; set++) {
        const double* anu = COL(s.anu, set);
        S ai = (S)anu[i];
        S d2c[4], d4c[4];
#pragma unroll
        for (int f = 0; f < 4; f++) {
            S e2 = (S)P.co2 * mx2(ai, (S)anu[nb[f]]);
            S e4 = mx2(S(0.0), (S)P.co4 - e2);
            d2c[f] = e2 * d24nc[f];
            d4c[f] = e4 * d24nc[f];
        }
#pragma unroll
        for (int k = 5 * set; k < 5 * set + 5; k++) {
            const double* cn = COL(s.cn, k);
            const double* dq = COL(s.d2q, k);
            S ci = (S)cn[i], qi = (S)dq[i];
            S d2 = d2c[0] * ((S)cn[nb[0]] - ci) + d2c[1] * ((S)cn[nb[1]] - ci) +
                   d2c[2] * ((S)cn[nb[2]] - ci) + d2c[3] * ((S)cn[nb[3]] - ci);
            S d4 = d4c[0] * ((S)dq[nb[0]] - qi) + d4c[1] * ((S)dq[nb[1]] - qi) +
                   d4c[2] * ((S)dq[nb[2]] - qi) + d4c[3] * ((S)dq[nb[3]] - qi);
            out[k] = d2 - d4;
        }
    }
    // all stores after all loads (see k_smooth1)
#pragma unroll
    for (int k = 0; k < 10; k++) COL(s.d24, k)[i] = out[k];
    return bad;
}

__device__ __forceinline__ void k_smooth2_body(DevMesh m, DevState<R> s, DevParams P, int bid) {
    int i = bid * blockDim.x + threadIdx.x;
    const bool valid = i < m.neles;
    if (!valid) i = m.neles - 1;      // keep the warp whole for the vote below
    if constexpr (HP_FAST(8)) {
        unsigned bad = 0;
        if (valid) bad = smooth2_body<1>(m, s, P, i);
        if (__any_sync(0xffffffffu, bad) && valid) smooth2_body<0>(m, s, P, i);
    } else {
        if (valid) smooth2_body<0>(m, s, P, i);
    }
}
__global__ void __launch_bounds__(512) k_smooth2(DevMesh m, DevState<R> s, DevParams P) {
    k_smooth2_body(m, s, P, blockIdx.x);
}

// Cells whose gradients and limiter are evaluated: active cells and the
// first halo layer of a partition part (iblank HP_IBLANK_HALO1), which its
// owner evaluates the same way; the halo is never RK-updated.
__device__ __forceinline__ bool grad_cell(int ib) { return ib == 1 || ib == HP_IBLANK_HALO1; }

// ---------------------------------------------------------------------------
// LSQ gradients (src/sr_derivative.F90:45-322) fused with the
// Venkatakrishnan limiter (src/sr_VK.F90:32-272).  grad_cell() cells.
// FPR: read the primitives in R (the float copy of the FP32-arithmetic
// variants) instead of the FP64 columns; false on aliased meshes.
// FP64 wall layers of the FP32 variants: a face whose two cells are layer
// cells (or a layer cell's boundary face) feeds only FP64 kernels, so the
// FP32 face kernels skip it.
__device__ __forceinline__ bool wall_face(const DevMesh& m, int i, int f) {
    if (sizeof(R) == sizeof(double) || m.nwall == 0 || !ldg(m.wclass + i)) return false;
    const int j = ldg(COL(m.nc, f) + i);
    return j >= m.neles || ldg(m.wclass + j) != 0;
}

template <bool FPR>
__device__ __forceinline__ void k_grad_body(DevMesh m, DevState<R> s, DevParams P, int bid) {
    using PT = typename std::conditional<FPR, R, double>::type;
    const PT* const prb = reinterpret_cast<const PT*>(FPR ? (const void*)s.prr : (const void*)s.pr);
    int i = bid * blockDim.x + threadIdx.x;
    if (i >= m.neles) return;
    if (!grad_cell(ldg(m.iblank + i))) return;
    // FP64 wall layers: no FP32 face reads the gradients of a layer cell
    // whose neighbours are all layer cells (class 2)
    if (sizeof(R) != sizeof(double) && m.nwall > 0 && ldg(m.wclass + i) == 2) return;
    int n[4];
#pragma unroll
    for (int f = 0; f < 4; f++) n[f] = ldg(COL(m.nc, f) + i);
    const double x0 = ldg(m.xc + i), y0 = ldg(m.yc + i), z0 = ldg(m.zc + i);
    R xa[4], ya[4], za[4];
#pragma unroll
    for (int f = 0; f < 4; f++) {
        if (FPR && HP_DXN_TABLE) {
            // the centroid differences, formed at set-up (the same subtraction)
            xa[f] = (R)ldg(COL(m.dxn, 3 * f) + i);
            ya[f] = (R)ldg(COL(m.dxn, 3 * f + 1) + i);
            za[f] = (R)ldg(COL(m.dxn, 3 * f + 2) + i);
        } else {
            xa[f] = (R)(ldg(m.xc + n[f]) - x0);
            ya[f] = (R)(ldg(m.yc + n[f]) - y0);
            za[f] = (R)(ldg(m.zc + n[f]) - z0);
        }
    }
    // geometry-only terms (wt, a1..b3, dnr of src/sr_derivative.F90:163-176,
    // 255), evaluated once at set-up with the same expressions
    R wt[4], rw[4];
#define DW(x, f) div_rn((x), wt[f], rw[f])
#if HP_LSQ_TABLE
#pragma unroll
    for (int f = 0; f < 4; f++) { wt[f] = (R)ldg(COL(m.lsqa, f) + i); rw[f] = rcp(wt[f]); }
    const R a1 = (R)ldg(COL(m.lsqa, 4) + i), a2 = (R)ldg(COL(m.lsqa, 5) + i), a3 = (R)ldg(COL(m.lsqa, 6) + i);
    const R b1 = (R)ldg(COL(m.lsqa, 7) + i), b2 = (R)ldg(COL(m.lsqa, 8) + i), b3 = (R)ldg(COL(m.lsqa, 9) + i);
    const R dnr = (R)ldg(COL(m.lsqa, 10) + i);
#else
#pragma unroll
    for (int f = 0; f < 4; f++) { wt[f] = xa[f] * xa[f] + ya[f] * ya[f] + za[f] * za[f]; rw[f] = rcp(wt[f]); }
    const R a1 = DW(xa[0] * xa[0], 0) + DW(xa[1] * xa[1], 1) + DW(xa[2] * xa[2], 2) + DW(xa[3] * xa[3], 3);
    const R a2 = DW(ya[0] * ya[0], 0) + DW(ya[1] * ya[1], 1) + DW(ya[2] * ya[2], 2) + DW(ya[3] * ya[3], 3);
    const R a3 = DW(za[0] * za[0], 0) + DW(za[1] * za[1], 1) + DW(za[2] * za[2], 2) + DW(za[3] * za[3], 3);
    const R b1 = DW(xa[0] * ya[0], 0) + DW(xa[1] * ya[1], 1) + DW(xa[2] * ya[2], 2) + DW(xa[3] * ya[3], 3);
    const R b2 = DW(xa[0] * za[0], 0) + DW(xa[1] * za[1], 1) + DW(xa[2] * za[2], 2) + DW(xa[3] * za[3], 3);
    const R b3 = DW(za[0] * ya[0], 0) + DW(za[1] * ya[1], 1) + DW(za[2] * ya[2], 2) + DW(za[3] * ya[3], 3);
    const R dnr = det3(a1, b1, b2, b1, a2, b3, b2, b3, a3);
#endif
    const R rdnr = rcp(dnr);
    // fields in the order of the stored gradient columns, then rog, rop
    const int pcol[13] = {P_UG, P_VG, P_WG, P_TG, P_UP, P_VP, P_WP, P_TP, P_PG, P_PP, P_PHIG, P_ROG, P_ROP};
    R gv[13][3];
#pragma unroll
    for (int v = 0; v < 13; v++) {
        R qa, qb, qc, qd;
        if (FPR && pcol[v] == P_PHIG) {
            // alpha_g differences from the FP64 primitives: near alpha_g = 1
            // the FP32 copies differ by whole ulps (6e-8), as much as a trace
            // alpha_p = 1 - alpha_g itself, whose reconstruction uses this
            // gradient
            const double* q = COL(s.pr, P_PHIG);
            const double qi = ldg(q + i);
            qa = (R)(ldg(q + n[0]) - qi); qb = (R)(ldg(q + n[1]) - qi);
            qc = (R)(ldg(q + n[2]) - qi); qd = (R)(ldg(q + n[3]) - qi);
        } else {
            const PT* q = COL(prb, pcol[v]);
            PT qi = ldg(q + i);
            qa = (R)(ldg(q + n[0]) - qi); qb = (R)(ldg(q + n[1]) - qi);
            qc = (R)(ldg(q + n[2]) - qi); qd = (R)(ldg(q + n[3]) - qi);
        }
        R c1 = DW(qa * xa[0], 0) + DW(qb * xa[1], 1) + DW(qc * xa[2], 2) + DW(qd * xa[3], 3);
        R c2;
        if (v == 7)   // cTp2 lacks the /wt4 (src/sr_derivative.F90:225)
            c2 = DW(qa * ya[0], 0) + DW(qb * ya[1], 1) + DW(qc * ya[2], 2) + qd * ya[3];
        else
            c2 = DW(qa * ya[0], 0) + DW(qb * ya[1], 1) + DW(qc * ya[2], 2) + DW(qd * ya[3], 3);
        R c3 = DW(qa * za[0], 0) + DW(qb * za[1], 1) + DW(qc * za[2], 2) + DW(qd * za[3], 3);
        gv[v][0] = div_rn(det3(c1, c2, c3, b1, a2, b3, b2, b3, a3), dnr, rdnr);
        gv[v][1] = div_rn(det3(a1, b1, b2, c1, c2, c3, b2, b3, a3), dnr, rdnr);
        gv[v][2] = div_rn(det3(a1, b1, b2, b1, a2, b3, c1, c2, c3), dnr, rdnr);
        // stored at once (the inputs are read through the read-only path,
        // so the stores do not order them); the limiter keeps 8, 9, 11, 12
        if (v < 11) {
            COL(s.gr, 3 * v + 0)[i] = gv[v][0];
            COL(s.gr, 3 * v + 1)[i] = gv[v][1];
            COL(s.gr, 3 * v + 2)[i] = gv[v][2];
        }
    }
    // limiter: phi_i = min over {pg, pp, rog, rop} x 4 faces
    const R epssq = (R)ldg(m.eps2 + i);
    R fx[4], fy[4], fz[4];
#pragma unroll
    for (int f = 0; f < 4; f++) {
        fx[f] = (R)(ldg(COL(m.fch, f) + i) - x0);
        fy[f] = (R)(ldg(COL(m.fch, 4 + f) + i) - y0);
        fz[f] = (R)(ldg(COL(m.fch, 8 + f) + i) - z0);
    }
    const int lv[4] = {8, 9, 11, 12};   // pg, pp, rog, rop rows of gv
    R phi = R(0);
#pragma unroll
    for (int t = 0; t < 4; t++) {
        const PT* q = COL(prb, pcol[lv[t]]);
        PT qi = ldg(q + i), q0 = ldg(q + n[0]), q1 = ldg(q + n[1]), q2 = ldg(q + n[2]), q3 = ldg(q + n[3]);
        PT vmax = mx2(mx2(mx2(mx2(qi, q0), q1), q2), q3);
        PT vmin = mn2(mn2(mn2(mn2(qi, q0), q1), q2), q3);
        R dmax = (R)(vmax - qi), dmin = (R)(vmin - qi);
        R gx = gv[lv[t]][0], gy = gv[lv[t]][1], gz = gv[lv[t]][2];
#pragma unroll
        for (int f = 0; f < 4; f++) {
            R d = fx[f] * gx + fy[f] * gy + fz[f] * gz;
            R ph;
            if (d > R(0)) ph = fvenkat(dmax, d, epssq);
            else if (d < R(0)) ph = fvenkat(dmin, d, epssq);
            else ph = R(1);
            phi = (t == 0 && f == 0) ? ph : mn2(phi, ph);
        }
    }
    s.phi[i] = (double)phi;
}
template <bool FPR>
__global__ void __launch_bounds__(128) k_grad(DevMesh m, DevState<R> s, DevParams P) {
    k_grad_body<FPR>(m, s, P, blockIdx.x);
}

// ---------------------------------------------------------------------------
// One face of cell i: MUSCL reconstruction, phase blending and HLLC-Batten
// (src/sr_hllcbatten.F90:79-529).  Wall faces return the pressure terms.
struct FaceOut {
    R F[10];
    R w[6];
    bool wall, takeg, takep;
};

template <int F>
__device__ __forceinline__ void blend_phases_r(const DevParams& P, R& phig, R& phip, R& ug, R& vg,
                                               R& wg, R& tg, R& pg, R& up, R& vp, R& wp, R& tp,
                                               R& pp, unsigned& bad) {
    const R emin = (R)P.emin, emax = (R)P.emax;
    if (phig < emin) {
        phig = emin; phip = R(1) - phig;
        ug = up; vg = vp; wg = wp; tg = tp; pg = pp;
    }
    if (phip < emin) {
        phip = emin; phig = R(1) - phip;
        up = ug; vp = vg; wp = wg; tp = tg; pp = pg;
    }
    if (phig >= emin && phig <= emax) {
        R psig = mdiv<F>(phig - emin, emax - emin, (R)P.r_emm, bad);
        R f = -(psig * psig * (R(2) * psig - R(3)));
        ug = f * ug + (R(1) - f) * up; vg = f * vg + (R(1) - f) * vp;
        wg = f * wg + (R(1) - f) * wp; tg = f * tg + (R(1) - f) * tp;
        pg = f * pg + (R(1) - f) * pp;
    }
    if (phip >= emin && phip <= emax) {
        R psig = mdiv<F>(phip - emin, emax - emin, (R)P.r_emm, bad);
        R f = -(psig * psig * (R(2) * psig - R(3)));
        up = f * up + (R(1) - f) * ug; vp = f * vp + (R(1) - f) * vg;
        wp = f * wp + (R(1) - f) * wg; tp = f * tp + (R(1) - f) * tg;
        pp = f * pp + (R(1) - f) * pg;
    }
}

// HLLC-Zien for one face (src/sr_hllczien.F90:348-487): wave speeds over
// both phases, a mixture contact speed, and one branch for all ten fluxes.
// takeg = takep = whether a branch was taken (NaN states take none).
template <int F>
__device__ __forceinline__ void zien_flux(FaceOut& o, unsigned& bad, R area, R enx, R eny, R enz,
                                          R phigL, R phipL, R rogL, R ropL, R ugL, R vgL, R wgL, R upL, R vpL,
                                          R wpL, R pgL, R ppL, R egL, R hgL, R qgL, R agL, R epL, R hpL, R qpL,
                                          R apL, R phigR, R phipR, R rogR, R ropR, R ugR, R vgR, R wgR, R upR,
                                          R vpR, R wpR, R pgR, R ppR, R egR, R hgR, R qgR, R agR, R epR, R hpR,
                                          R qpR, R apR) {
    const R eps8 = (R)(double)1.0e-8f, eps6 = (R)(double)1.0e-6f;
    // DMIN1 / DMAX1 of five arguments, left to right
    const R sl = mn2(mn2(mn2(mn2(qgL - agL, qpL - apL), qgR - agR), qpR - apR), eps8);
    const R sr = mx2(mx2(mx2(mx2(qgL + agL, qpL + apL), qgR + agR), qpR + apR), eps8);
    const R rol = phigL * rogL + phipL * ropL;
    const R roql = phigL * rogL * qgL + phipL * ropL * qpL;
    const R ql = roql / rol;
    const R prl = phigL * pgL + phipL * ppL;
    const R ror = phigR * rogR + phipR * ropR;
    const R roqr = phigR * rogR * qgR + phipR * ropR * qpR;
    const R qr = roqr / ror;
    const R prr = phigR * pgR + phipR * ppR;
    const R sstar = (prr - prl + roql * (sl - ql) - roqr * (sr - qr)) / ((rol * (sl - ql) - ror * (sr - qr)) + eps8);
    const R pgstar = mx2(pgL + rogL * (qgL - sl) * (qgL - sstar), eps6 * mn2(pgL, pgR));
    const R ppstar = mx2(ppL + ropL * (qpL - sl) * (qpL - sstar), eps6 * mn2(ppL, ppR));
    const int br = (sl >= R(0)) ? 1 : (sl <= R(0) && sstar > R(0)) ? 2
                   : (sstar <= R(0) && sr >= R(0)) ? 3 : (sr <= R(0)) ? 4 : 0;
    o.takeg = o.takep = br != 0;
    if (br == 1 || br == 2) {
        R cn[10], fx[10];
        cn[0] = phigL * rogL; cn[1] = phigL * rogL * ugL; cn[2] = phigL * rogL * vgL;
        cn[3] = phigL * rogL * wgL; cn[4] = phigL * rogL * egL;
        cn[5] = phipL * ropL; cn[6] = phipL * ropL * upL; cn[7] = phipL * ropL * vpL;
        cn[8] = phipL * ropL * wpL; cn[9] = phipL * ropL * epL;
        fx[0] = phigL * rogL * qgL;
        fx[1] = phigL * rogL * qgL * ugL + phigL * pgL * enx;
        fx[2] = phigL * rogL * qgL * vgL + phigL * pgL * eny;
        fx[3] = phigL * rogL * qgL * wgL + phigL * pgL * enz;
        fx[4] = phigL * rogL * qgL * hgL;
        fx[5] = phipL * ropL * qpL;
        fx[6] = phipL * ropL * qpL * upL + phipL * ppL * enx;
        fx[7] = phipL * ropL * qpL * vpL + phipL * ppL * eny;
        fx[8] = phipL * ropL * qpL * wpL + phipL * ppL * enz;
        fx[9] = phipL * ropL * qpL * hpL;
        if (br == 1) {
#pragma unroll
            for (int k = 0; k < 10; k++) o.F[k] = fx[k] * area;
        } else {
            const R dnr = (sstar - sl) + eps6;
            const R rd = mrcp<F>(dnr, bad);
            R cs[10];
            cs[0] = mdiv<F>((qgL - sl) * cn[0], dnr, rd, bad);
            cs[1] = mdiv<F>((qgL - sl) * cn[1] + phigL * (pgL * enx - pgstar * enx), dnr, rd, bad);
            cs[2] = mdiv<F>((qgL - sl) * cn[2] + phigL * (pgL * eny - pgstar * eny), dnr, rd, bad);
            cs[3] = mdiv<F>((qgL - sl) * cn[3] + phigL * (pgL * enz - pgstar * enz), dnr, rd, bad);
            cs[4] = mdiv<F>((qgL - sl) * cn[4] + phigL * (pgL * qgL - pgstar * sstar), dnr, rd, bad);
            cs[5] = mdiv<F>((qpL - sl) * cn[5], dnr, rd, bad);
            cs[6] = mdiv<F>((qpL - sl) * cn[6] + phipL * (ppL * enx - ppstar * enx), dnr, rd, bad);
            cs[7] = mdiv<F>((qpL - sl) * cn[7] + phipL * (ppL * eny - ppstar * eny), dnr, rd, bad);
            cs[8] = mdiv<F>((qpL - sl) * cn[8] + phipL * (ppL * enz - ppstar * enz), dnr, rd, bad);
            cs[9] = mdiv<F>((qpL - sl) * cn[9] + phipL * (ppL * qpL - ppstar * sstar), dnr, rd, bad);
#pragma unroll
            for (int k = 0; k < 10; k++) o.F[k] = (fx[k] + sl * (cs[k] - cn[k])) * area;
        }
    } else if (br == 4 || br == 3) {
        R cn[10], fx[10];
        cn[0] = phigR * rogR; cn[1] = phigR * rogR * ugR; cn[2] = phigR * rogR * vgR;
        cn[3] = phigR * rogR * wgR; cn[4] = phigR * rogR * egR;
        cn[5] = phipR * ropR; cn[6] = phipR * ropR * upR; cn[7] = phipR * ropR * vpR;
        cn[8] = phipR * ropR * wpR; cn[9] = phipR * ropR * epR;
        fx[0] = phigR * rogR * qgR;
        fx[1] = phigR * rogR * qgR * ugR + phigR * pgR * enx;
        fx[2] = phigR * rogR * qgR * vgR + phigR * pgR * eny;
        fx[3] = phigR * rogR * qgR * wgR + phigR * pgR * enz;
        fx[4] = phigR * rogR * qgR * hgR;
        fx[5] = phipR * ropR * qpR;
        fx[6] = phipR * ropR * qpR * upR + phipR * ppR * enx;
        fx[7] = phipR * ropR * qpR * vpR + phipR * ppR * eny;
        fx[8] = phipR * ropR * qpR * wpR + phipR * ppR * enz;
        fx[9] = phipR * ropR * qpR * hpR;
        if (br == 4) {
#pragma unroll
            for (int k = 0; k < 10; k++) o.F[k] = fx[k] * area;
        } else {
            const R dnr = (sstar - sr) + eps6;
            const R rd = mrcp<F>(dnr, bad);
            R cs[10];
            cs[0] = mdiv<F>((qgR - sr) * cn[0], dnr, rd, bad);
            cs[1] = mdiv<F>((qgR - sr) * cn[1] + phigR * (pgR * enx - pgstar * enx), dnr, rd, bad);
            cs[2] = mdiv<F>((qgR - sr) * cn[2] + phigR * (pgR * eny - pgstar * eny), dnr, rd, bad);
            cs[3] = mdiv<F>((qgR - sr) * cn[3] + phigR * (pgR * enz - pgstar * enz), dnr, rd, bad);
            cs[4] = mdiv<F>((qgR - sr) * cn[4] + phigR * (pgR * qgR - pgstar * sstar), dnr, rd, bad);
            cs[5] = mdiv<F>((qpR - sr) * cn[5], dnr, rd, bad);
            cs[6] = mdiv<F>((qpR - sr) * cn[6] + phipR * (ppR * enx - ppstar * enx), dnr, rd, bad);
            cs[7] = mdiv<F>((qpR - sr) * cn[7] + phipR * (ppR * eny - ppstar * eny), dnr, rd, bad);
            cs[8] = mdiv<F>((qpR - sr) * cn[8] + phipR * (ppR * enz - ppstar * enz), dnr, rd, bad);
            cs[9] = mdiv<F>((qpR - sr) * cn[9] + phipR * (ppR * qpR - ppstar * sstar), dnr, rd, bad);
#pragma unroll
            for (int k = 0; k < 10; k++) o.F[k] = (fx[k] + sr * (cs[k] - cn[k])) * area;
        }
    }
}

// face-state loads through the read-only data path (1) or plain (0)
// Asynchronous global-to-shared copies: 16 bytes through L2 only (the tail
// prefetch of the four-lane flux kernel), 8 bytes through L1 (the staged
// four-lane gradient kernel).
#ifndef HP_FLUX4_PREFETCH
#define HP_FLUX4_PREFETCH 0
#endif
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
enum { LIM_LD = 128, LIMC_N = 13, LIMC_LD = 32 };

#ifndef HP_FACE_LDG
#define HP_FACE_LDG 1
#endif
// (NC = false: plain loads, for the fused step, which writes these arrays)
#define PLD(p) ((HP_FACE_LDG && NC) ? ldg(p) : *(p))
// F selects the division form (see mdiv); bad collects its out-of-range flag.
// Z selects the face flux: 0 HLLC-Batten (src/sr_hllcbatten.F90:338-529),
// 1 HLLC-Zien (src/sr_hllczien.F90:348-487), 2 the Jameson central flux
// (src/sr_jameson.F90:126-262).
template <int F, int Z, class PT, bool NC = true>
__device__ __forceinline__ void face_eval(const DevMesh& m, const DevState<R>& s, const DevParams& P,
                                          int i, int f, FaceOut& o, unsigned& bad, const PT* pr) {
    const int neigh = ldg(COL(m.nc, f) + i);
    const unsigned kind = (ldg(m.fk + i) >> (4 * f)) & 0xFu;
    const double scxd = ldg(COL(m.sc, 3 * f) + i), scyd = ldg(COL(m.sc, 3 * f + 1) + i),
                 sczd = ldg(COL(m.sc, 3 * f + 2) + i);
    const R scx = (R)scxd, scy = (R)scyd, scz = (R)sczd;
    const R area = sqrt(scx * scx + scy * scy + scz * scz);
    const R rarea = mrcp<F>(area, bad);
    const R enx = mdiv<F>(scx, area, rarea, bad), eny = mdiv<F>(scy, area, rarea, bad), enz = mdiv<F>(scz, area, rarea, bad);
    R ugL = (R)PLD(COL(pr, P_UG) + i), vgL = (R)PLD(COL(pr, P_VG) + i), wgL = (R)PLD(COL(pr, P_WG) + i);
    R tgL = (R)PLD(COL(pr, P_TG) + i), phigL = (R)PLD(COL(pr, P_PHIG) + i);
    R upL = (R)PLD(COL(pr, P_UP) + i), vpL = (R)PLD(COL(pr, P_VP) + i), wpL = (R)PLD(COL(pr, P_WP) + i);
    R tpL = (R)PLD(COL(pr, P_TP) + i), pgL = (R)PLD(COL(pr, P_PG) + i), ppL = (R)PLD(COL(pr, P_PP) + i);
    R ugR = (R)PLD(COL(pr, P_UG) + neigh), vgR = (R)PLD(COL(pr, P_VG) + neigh), wgR = (R)PLD(COL(pr, P_WG) + neigh);
    R tgR = (R)PLD(COL(pr, P_TG) + neigh), phigR = (R)PLD(COL(pr, P_PHIG) + neigh);
    R upR = (R)PLD(COL(pr, P_UP) + neigh), vpR = (R)PLD(COL(pr, P_VP) + neigh), wpR = (R)PLD(COL(pr, P_WP) + neigh);
    R tpR = (R)PLD(COL(pr, P_TP) + neigh), pgR = (R)PLD(COL(pr, P_PG) + neigh), ppR = (R)PLD(COL(pr, P_PP) + neigh);
    // alpha_p.  The reference forms it as 1 - alpha_g after reconstruction
    // (src/sr_hllcbatten.F90:226-227), which the FP64 variants keep.  In FP32
    // that difference loses everything where the water is a trace: with
    // alpha_g = 1 - 1e-6 one FP32 ulp of alpha_g is 6% of alpha_p.  The FP32
    // variants therefore start from the cell's own alpha_p (recovered in FP64)
    // and subtract the reconstruction increment of alpha_g, which is the same
    // quantity mathematically and keeps alpha_p to FP32 relative precision.
    // With dispersed phases alpha_g + alpha_p = 1 - their fractions, and the
    // reference still takes 1 - alpha_g: formed here in FP64 from alpha_g.
    R phipL = R(0), phipR = R(0);
    if constexpr (sizeof(R) == 4) {
        if (P.five_phase) {
            phipL = (R)(1.0 - PLD(COL(s.pr, P_PHIG) + i));
            phipR = (R)(1.0 - PLD(COL(s.pr, P_PHIG) + neigh));
        } else {
            phipL = (R)PLD(COL(pr, P_PHIP) + i);
            phipR = (R)PLD(COL(pr, P_PHIP) + neigh);
        }
    }
    if constexpr (Z == 2) {
        // Jameson central flux (src/sr_jameson.F90:126-262): the two cells'
        // own values, no reconstruction and no phase blending, the densities
        // of the primitive recovery; the face flux is the mean of the two
        // sides' physical fluxes times the area, so both phases always take it
        if constexpr (sizeof(R) != 4) {
            phipL = R(1) - phigL;
            phipR = R(1) - phigR;
        }
        o.wall = (kind & FK_WALL) != 0;
        o.takeg = o.takep = !o.wall;
        if (o.wall) {   // :185-191
            o.w[0] = phigL * pgL * enx * area;
            o.w[1] = phigL * pgL * eny * area;
            o.w[2] = phigL * pgL * enz * area;
            o.w[3] = phipL * ppL * enx * area;
            o.w[4] = phipL * ppL * eny * area;
            o.w[5] = phipL * ppL * enz * area;
            return;
        }
        const R rrg = (R)P.rrg, gamag = (R)P.gamag, gamap = (R)P.gamap, pinf = (R)P.pinf, cpp = (R)P.cpp;
        const R rgm1 = (R)P.r_gm1, rgamap = (R)P.r_gamap;
        const R rogL = (R)PLD(COL(pr, P_ROG) + i), ropL = (R)PLD(COL(pr, P_ROP) + i);
        const R rogR = (R)PLD(COL(pr, P_ROG) + neigh), ropR = (R)PLD(COL(pr, P_ROP) + neigh);
        const R rrogL = mrcp<F>(rogL, bad), rrogR = mrcp<F>(rogR, bad);
        const R rropL = mrcp<F>(ropL, bad), rropR = mrcp<F>(ropR, bad);
        // :194-212 (the sound speeds formed there enter no flux)
        const R egL = mdiv<F>(rrg * tgL, gamag - R(1), rgm1, bad) + R(0.5) * (ugL * ugL + vgL * vgL + wgL * wgL);
        const R hgL = egL + mdiv<F>(pgL, rogL, rrogL, bad);
        const R qgL = ugL * enx + vgL * eny + wgL * enz;
        const R egR = mdiv<F>(rrg * tgR, gamag - R(1), rgm1, bad) + R(0.5) * (ugR * ugR + vgR * vgR + wgR * wgR);
        const R hgR = egR + mdiv<F>(pgR, rogR, rrogR, bad);
        const R qgR = ugR * enx + vgR * eny + wgR * enz;
        const R epL = mdiv<F>(cpp * tpL, gamap, rgamap, bad) + mdiv<F>(pinf, ropL, rropL, bad) +
                      R(0.5) * (upL * upL + vpL * vpL + wpL * wpL);
        const R hpL = epL + mdiv<F>(ppL, ropL, rropL, bad);
        const R qpL = upL * enx + vpL * eny + wpL * enz;
        const R epR = mdiv<F>(cpp * tpR, gamap, rgamap, bad) + mdiv<F>(pinf, ropR, rropR, bad) +
                      R(0.5) * (upR * upR + vpR * vpR + wpR * wpR);
        const R hpR = epR + mdiv<F>(ppR, ropR, rropR, bad);
        const R qpR = upR * enx + vpR * eny + wpR * enz;
        // :216-261
        o.F[0] = (phigL * rogL * qgL + phigR * rogR * qgR) * R(0.5) * area;
        o.F[1] = ((phigL * rogL * qgL * ugL + phigL * pgL * enx) + (phigR * rogR * qgR * ugR + phigR * pgR * enx)) *
                 R(0.5) * area;
        o.F[2] = ((phigL * rogL * qgL * vgL + phigL * pgL * eny) + (phigR * rogR * qgR * vgR + phigR * pgR * eny)) *
                 R(0.5) * area;
        o.F[3] = ((phigL * rogL * qgL * wgL + phigL * pgL * enz) + (phigR * rogR * qgR * wgR + phigR * pgR * enz)) *
                 R(0.5) * area;
        o.F[4] = (phigL * rogL * qgL * hgL + phigR * rogR * qgR * hgR) * R(0.5) * area;
        o.F[5] = (phipL * ropL * qpL + phipR * ropR * qpR) * R(0.5) * area;
        o.F[6] = ((phipL * ropL * qpL * upL + phipL * ppL * enx) + (phipR * ropR * qpR * upR + phipR * ppR * enx)) *
                 R(0.5) * area;
        o.F[7] = ((phipL * ropL * qpL * vpL + phipL * ppL * eny) + (phipR * ropR * qpR * vpR + phipR * ppR * eny)) *
                 R(0.5) * area;
        o.F[8] = ((phipL * ropL * qpL * wpL + phipL * ppL * enz) + (phipR * ropR * qpR * wpR + phipR * ppR * enz)) *
                 R(0.5) * area;
        o.F[9] = (phipL * ropL * qpL * hpL + phipR * ropR * qpR * hpR) * R(0.5) * area;
        return;
    }
    if (P.myorder == 2 && (kind & FK_RECON)) {
        const R phimin = (R)mn2(PLD(s.phi + i), PLD(s.phi + neigh));
        const double xf = ldg(COL(m.fch, f) + i), yf = ldg(COL(m.fch, 4 + f) + i),
                     zf = ldg(COL(m.fch, 8 + f) + i);
        const R xf0 = (R)(xf - ldg(m.xc + i)), yf0 = (R)(yf - ldg(m.yc + i)), zf0 = (R)(zf - ldg(m.zc + i));
        const R xfn = (R)(xf - ldg(m.xc + neigh)), yfn = (R)(yf - ldg(m.yc + neigh)),
                zfn = (R)(zf - ldg(m.zc + neigh));
        const R* g = s.gr;
#define REC(v, X, Y, Z, G, c) \
    v = v + phimin * (X * PLD(COL(g, G) + c) + Y * PLD(COL(g, G + 1) + c) + Z * PLD(COL(g, G + 2) + c))
        if constexpr (sizeof(R) == 4) {
            const R dL = xf0 * PLD(COL(g, G_PHIG) + i) + yf0 * PLD(COL(g, G_PHIG + 1) + i) +
                         zf0 * PLD(COL(g, G_PHIG + 2) + i);
            const R dR = xfn * PLD(COL(g, G_PHIG) + neigh) + yfn * PLD(COL(g, G_PHIG + 1) + neigh) +
                         zfn * PLD(COL(g, G_PHIG + 2) + neigh);
            phigL = phigL + phimin * dL; phipL = phipL - phimin * dL;
            phigR = phigR + phimin * dR; phipR = phipR - phimin * dR;
        } else {
            REC(phigL, xf0, yf0, zf0, G_PHIG, i);
            REC(phigR, xfn, yfn, zfn, G_PHIG, neigh);
        }
        REC(ugL, xf0, yf0, zf0, G_UG, i);
        REC(vgL, xf0, yf0, zf0, G_VG, i); REC(wgL, xf0, yf0, zf0, G_WG, i);
        REC(tgL, xf0, yf0, zf0, G_TG, i); REC(pgL, xf0, yf0, zf0, G_PG, i);
        REC(ugR, xfn, yfn, zfn, G_UG, neigh);
        REC(vgR, xfn, yfn, zfn, G_VG, neigh); REC(wgR, xfn, yfn, zfn, G_WG, neigh);
        REC(tgR, xfn, yfn, zfn, G_TG, neigh); REC(pgR, xfn, yfn, zfn, G_PG, neigh);
        REC(upL, xf0, yf0, zf0, G_UP, i); REC(vpL, xf0, yf0, zf0, G_VP, i);
        REC(wpL, xf0, yf0, zf0, G_WP, i); REC(tpL, xf0, yf0, zf0, G_TP, i);
        REC(ppL, xf0, yf0, zf0, G_PP, i);
        REC(upR, xfn, yfn, zfn, G_UP, neigh); REC(vpR, xfn, yfn, zfn, G_VP, neigh);
        REC(wpR, xfn, yfn, zfn, G_WP, neigh); REC(tpR, xfn, yfn, zfn, G_TP, neigh);
        REC(ppR, xfn, yfn, zfn, G_PP, neigh);
#undef REC
    }
    const R rrg = (R)P.rrg, gamag = (R)P.gamag, gamap = (R)P.gamap, pinf = (R)P.pinf, cpp = (R)P.cpp;
    if constexpr (sizeof(R) != 4) {
        phipL = R(1) - phigL;
        phipR = R(1) - phigR;
    }
    blend_phases_r<F>(P, phigL, phipL, ugL, vgL, wgL, tgL, pgL, upL, vpL, wpL, tpL, ppL, bad);
    R rogL = pgL / (rrg * tgL);
    R ropL = gamap * (ppL + pinf) / ((gamap - R(1)) * cpp * tpL);
    blend_phases_r<F>(P, phigR, phipR, ugR, vgR, wgR, tgR, pgR, upR, vpR, wpR, tpR, ppR, bad);
    R rogR = pgR / (rrg * tgR);
    R ropR = gamap * (ppR + pinf) / ((gamap - R(1)) * cpp * tpR);
    o.wall = (kind & FK_WALL) != 0;
    if (o.wall) {
        o.w[0] = phigL * pgL * enx * area;
        o.w[1] = phigL * pgL * eny * area;
        o.w[2] = phigL * pgL * enz * area;
        o.w[3] = phipL * ppL * enx * area;
        o.w[4] = phipL * ppL * eny * area;
        o.w[5] = phipL * ppL * enz * area;
        o.takeg = o.takep = false;
        return;
    }
    const R eps8 = (R)(double)1.0e-8f, eps6 = (R)(double)1.0e-6f;
    const R rgm1 = (R)P.r_gm1, rgamap = (R)P.r_gamap;
    // the gas phase's wave speeds and HLLC first, then the liquid's: each
    // phase's quantities are live only while it is evaluated (the values and
    // their order of evaluation are those of src/sr_hllcbatten.F90:338-529)
    R egL = mdiv<F>(rrg * tgL, gamag - R(1), rgm1, bad) + R(0.5) * (ugL * ugL + vgL * vgL + wgL * wgL);
    const R rrogL = mrcp<F>(rogL, bad), rrogR = mrcp<F>(rogR, bad);
    R hgL = egL + mdiv<F>(pgL, rogL, rrogL, bad);
    R qgL = ugL * enx + vgL * eny + wgL * enz;
    R agL = sqrt(mdiv<F>(gamag * pgL, rogL, rrogL, bad));
    R egR = mdiv<F>(rrg * tgR, gamag - R(1), rgm1, bad) + R(0.5) * (ugR * ugR + vgR * vgR + wgR * wgR);
    R hgR = egR + mdiv<F>(pgR, rogR, rrogR, bad);
    R qgR = ugR * enx + vgR * eny + wgR * enz;
    R agR = sqrt(mdiv<F>(gamag * pgR, rogR, rrogR, bad));
#define HP_LIQUID_WAVES \
    const R rropL = mrcp<F>(ropL, bad), rropR = mrcp<F>(ropR, bad); \
    R epL = mdiv<F>(cpp * tpL, gamap, rgamap, bad) + mdiv<F>(pinf, ropL, rropL, bad) + \
            R(0.5) * (upL * upL + vpL * vpL + wpL * wpL); \
    R hpL = epL + mdiv<F>(ppL, ropL, rropL, bad); \
    R qpL = upL * enx + vpL * eny + wpL * enz; \
    R apL = sqrt(mdiv<F>(gamap * (ppL + pinf), ropL, rropL, bad)); \
    R epR = mdiv<F>(cpp * tpR, gamap, rgamap, bad) + mdiv<F>(pinf, ropR, rropR, bad) + \
            R(0.5) * (upR * upR + vpR * vpR + wpR * wpR); \
    R hpR = epR + mdiv<F>(ppR, ropR, rropR, bad); \
    R qpR = upR * enx + vpR * eny + wpR * enz; \
    R apR = sqrt(mdiv<F>(gamap * (ppR + pinf), ropR, rropR, bad));
    if constexpr (Z == 1) {
        HP_LIQUID_WAVES
        zien_flux<F>(o, bad, area, enx, eny, enz, phigL, phipL, rogL, ropL, ugL, vgL, wgL, upL, vpL, wpL, pgL,
                     ppL, egL, hgL, qgL, agL, epL, hpL, qpL, apL, phigR, phipR, rogR, ropR, ugR, vgR, wgR, upR,
                     vpR, wpR, pgR, ppR, egR, hgR, qgR, agR, epR, hpR, qpR, apR);
        return;
    }
    R sgl = mn2(mn2(qgL - agL, qgR - agR), eps8);
    R sgr = mx2(mx2(qgL + agL, qgR + agR), eps8);
    R sgstar = (pgR - pgL + rogL * qgL * (sgl - qgL) - rogR * qgR * (sgr - qgR)) /
               ((rogL * (sgl - qgL) - rogR * (sgr - qgR)) + eps8);
    R pgstar = mx2(pgL + rogL * (qgL - sgl) * (qgL - sgstar), eps6 * mn2(pgL, pgR));
    // gas phase
    {
        int br = (sgl > R(0)) ? 1 : (sgl <= R(0) && sgstar > R(0)) ? 2
                 : (sgstar <= R(0) && sgr >= R(0)) ? 3 : (sgr < R(0)) ? 4 : 0;
        o.takeg = br != 0;
        if (br == 1 || br == 2) {
            R cn0 = phigL * rogL, cn1 = phigL * rogL * ugL, cn2 = phigL * rogL * vgL;
            R cn3 = phigL * rogL * wgL, cn4 = phigL * rogL * egL;
            R fl0 = phigL * rogL * qgL;
            R fl1 = phigL * rogL * qgL * ugL + phigL * pgL * enx;
            R fl2 = phigL * rogL * qgL * vgL + phigL * pgL * eny;
            R fl3 = phigL * rogL * qgL * wgL + phigL * pgL * enz;
            R fl4 = phigL * rogL * qgL * hgL;
            if (br == 1) {
                o.F[0] = fl0 * area; o.F[1] = fl1 * area; o.F[2] = fl2 * area;
                o.F[3] = fl3 * area; o.F[4] = fl4 * area;
            } else {
                R dnrg = (sgstar - sgl) + eps6;
                const R rd = mrcp<F>(dnrg, bad);
                R cs0 = mdiv<F>((qgL - sgl) * cn0, dnrg, rd, bad);
                R cs1 = mdiv<F>((qgL - sgl) * cn1 + phigL * (pgL * enx - pgstar * enx), dnrg, rd, bad);
                R cs2 = mdiv<F>((qgL - sgl) * cn2 + phigL * (pgL * eny - pgstar * eny), dnrg, rd, bad);
                R cs3 = mdiv<F>((qgL - sgl) * cn3 + phigL * (pgL * enz - pgstar * enz), dnrg, rd, bad);
                R cs4 = mdiv<F>((qgL - sgl) * cn4 + phigL * (pgL * qgL - pgstar * sgstar), dnrg, rd, bad);
                o.F[0] = (fl0 + sgl * (cs0 - cn0)) * area;
                o.F[1] = (fl1 + sgl * (cs1 - cn1)) * area;
                o.F[2] = (fl2 + sgl * (cs2 - cn2)) * area;
                o.F[3] = (fl3 + sgl * (cs3 - cn3)) * area;
                o.F[4] = (fl4 + sgl * (cs4 - cn4)) * area;
            }
        } else if (br == 3 || br == 4) {
            R cn0 = phigR * rogR, cn1 = phigR * rogR * ugR, cn2 = phigR * rogR * vgR;
            R cn3 = phigR * rogR * wgR, cn4 = phigR * rogR * egR;
            R fr0 = phigR * rogR * qgR;
            R fr1 = phigR * rogR * qgR * ugR + phigR * pgR * enx;
            R fr2 = phigR * rogR * qgR * vgR + phigR * pgR * eny;
            R fr3 = phigR * rogR * qgR * wgR + phigR * pgR * enz;
            R fr4 = phigR * rogR * qgR * hgR;
            if (br == 4) {
                o.F[0] = fr0 * area; o.F[1] = fr1 * area; o.F[2] = fr2 * area;
                o.F[3] = fr3 * area; o.F[4] = fr4 * area;
            } else {
                R dnrg = (sgstar - sgr) + eps6;
                const R rd = mrcp<F>(dnrg, bad);
                R cs0 = mdiv<F>((qgR - sgr) * cn0, dnrg, rd, bad);
                R cs1 = mdiv<F>((qgR - sgr) * cn1 + phigR * (pgR * enx - pgstar * enx), dnrg, rd, bad);
                R cs2 = mdiv<F>((qgR - sgr) * cn2 + phigR * (pgR * eny - pgstar * eny), dnrg, rd, bad);
                R cs3 = mdiv<F>((qgR - sgr) * cn3 + phigR * (pgR * enz - pgstar * enz), dnrg, rd, bad);
                R cs4 = mdiv<F>((qgR - sgr) * cn4 + phigR * (pgR * qgR - pgstar * sgstar), dnrg, rd, bad);
                o.F[0] = (fr0 + sgr * (cs0 - cn0)) * area;
                o.F[1] = (fr1 + sgr * (cs1 - cn1)) * area;
                o.F[2] = (fr2 + sgr * (cs2 - cn2)) * area;
                o.F[3] = (fr3 + sgr * (cs3 - cn3)) * area;
                o.F[4] = (fr4 + sgr * (cs4 - cn4)) * area;
            }
        }
    }
    HP_LIQUID_WAVES
#undef HP_LIQUID_WAVES
    R spl = mn2(mn2(qpL - apL, qpR - apR), eps8);
    R spr = mx2(mx2(qpL + apL, qpR + apR), eps8);
    R spstar = (ppR - ppL + ropL * qpL * (spl - qpL) - ropR * qpR * (spr - qpR)) /
               ((ropL * (spl - qpL) - ropR * (spr - qpR)) + eps8);
    R ppstar = mx2(ppL + ropL * (qpL - spl) * (qpL - spstar), eps6 * mn2(ppL, ppR));
    // liquid phase
    {
        int br = (spl > R(0)) ? 1 : (spl <= R(0) && spstar > R(0)) ? 2
                 : (spstar <= R(0) && spr >= R(0)) ? 3 : (spr < R(0)) ? 4 : 0;
        o.takep = br != 0;
        if (br == 1 || br == 2) {
            R cn0 = phipL * ropL, cn1 = phipL * ropL * upL, cn2 = phipL * ropL * vpL;
            R cn3 = phipL * ropL * wpL, cn4 = phipL * ropL * epL;
            R fl0 = phipL * ropL * qpL;
            R fl1 = phipL * ropL * qpL * upL + phipL * ppL * enx;
            R fl2 = phipL * ropL * qpL * vpL + phipL * ppL * eny;
            R fl3 = phipL * ropL * qpL * wpL + phipL * ppL * enz;
            R fl4 = phipL * ropL * qpL * hpL;
            if (br == 1) {
                o.F[5] = fl0 * area; o.F[6] = fl1 * area; o.F[7] = fl2 * area;
                o.F[8] = fl3 * area; o.F[9] = fl4 * area;
            } else {
                R dnrp = (spstar - spl) + eps6;
                const R rd = mrcp<F>(dnrp, bad);
                R cs0 = mdiv<F>((qpL - spl) * cn0, dnrp, rd, bad);
                R cs1 = mdiv<F>((qpL - spl) * cn1 + phipL * (ppL * enx - ppstar * enx), dnrp, rd, bad);
                R cs2 = mdiv<F>((qpL - spl) * cn2 + phipL * (ppL * eny - ppstar * eny), dnrp, rd, bad);
                R cs3 = mdiv<F>((qpL - spl) * cn3 + phipL * (ppL * enz - ppstar * enz), dnrp, rd, bad);
                R cs4 = mdiv<F>((qpL - spl) * cn4 + phipL * (ppL * qpL - ppstar * spstar), dnrp, rd, bad);
                o.F[5] = (fl0 + spl * (cs0 - cn0)) * area;
                o.F[6] = (fl1 + spl * (cs1 - cn1)) * area;
                o.F[7] = (fl2 + spl * (cs2 - cn2)) * area;
                o.F[8] = (fl3 + spl * (cs3 - cn3)) * area;
                o.F[9] = (fl4 + spl * (cs4 - cn4)) * area;
            }
        } else if (br == 3 || br == 4) {
            R cn0 = phipR * ropR, cn1 = phipR * ropR * upR, cn2 = phipR * ropR * vpR;
            R cn3 = phipR * ropR * wpR, cn4 = phipR * ropR * epR;
            R fr0 = phipR * ropR * qpR;
            R fr1 = phipR * ropR * qpR * upR + phipR * ppR * enx;
            R fr2 = phipR * ropR * qpR * vpR + phipR * ppR * eny;
            R fr3 = phipR * ropR * qpR * wpR + phipR * ppR * enz;
            R fr4 = phipR * ropR * qpR * hpR;
            if (br == 4) {
                o.F[5] = fr0 * area; o.F[6] = fr1 * area; o.F[7] = fr2 * area;
                o.F[8] = fr3 * area; o.F[9] = fr4 * area;
            } else {
                R dnrp = (spstar - spr) + eps6;
                const R rd = mrcp<F>(dnrp, bad);
                R cs0 = mdiv<F>((qpR - spr) * cn0, dnrp, rd, bad);
                R cs1 = mdiv<F>((qpR - spr) * cn1 + phipR * (ppR * enx - ppstar * enx), dnrp, rd, bad);
                R cs2 = mdiv<F>((qpR - spr) * cn2 + phipR * (ppR * eny - ppstar * eny), dnrp, rd, bad);
                R cs3 = mdiv<F>((qpR - spr) * cn3 + phipR * (ppR * enz - ppstar * enz), dnrp, rd, bad);
                R cs4 = mdiv<F>((qpR - spr) * cn4 + phipR * (ppR * qpR - ppstar * spstar), dnrp, rd, bad);
                o.F[5] = (fr0 + spr * (cs0 - cn0)) * area;
                o.F[6] = (fr1 + spr * (cs1 - cn1)) * area;
                o.F[7] = (fr2 + spr * (cs2 - cn2)) * area;
                o.F[8] = (fr3 + spr * (cs3 - cn3)) * area;
                o.F[9] = (fr4 + spr * (cs4 - cn4)) * area;
            }
        }
    }
}

// Flux of the most recently evaluated face, in the reference's sequential
// cell order, whose wave branch was taken -- what the reference's FSTARA
// variables hold when a NaN state leaves every branch untaken.  Scans
// backwards from (i, f); falls back to the carry of the previous call.
template <int Z>
__device__ __noinline__ void stale_flux(const DevMesh& m, const DevState<R>& s, const DevParams& P,
                                        int i, int f, bool gas, R* out) {
    int cell = i, face = f - 1;
    for (int guard = 0; guard < (1 << 20); guard++) {
        if (face < 0) {
            cell--;
            while (cell >= 0 && ldg(m.iblank + cell) != 1) cell--;
            if (cell < 0) break;
            face = 3;
        }
        FaceOut o;
        unsigned bad_ = 0;
        face_eval<0, Z>(m, s, P, cell, face, o, bad_, s.pr);
        if (!o.wall && (gas ? o.takeg : o.takep)) {
            for (int k = 0; k < 5; k++) out[k] = o.F[(gas ? 0 : 5) + k];
            return;
        }
        face--;
    }
    for (int k = 0; k < 5; k++) out[k] = (R)s.s->fcarry[(gas ? 0 : 5) + k];
}

// Updates the stale-flux carry with the last taken face of the sweep; one
// thread, aliased meshes only.
template <int Z>
__global__ void k_flux_carry(DevMesh m, DevState<R> s, DevParams P) {
    R tmp[5];
    int last = m.neles - 1;
    while (last >= 0 && ldg(m.iblank + last) != 1) last--;
    if (last < 0) return;
    stale_flux<Z>(m, s, P, last, 4, true, tmp);
    for (int k = 0; k < 5; k++) s.s->fcarry[k] = (double)tmp[k];
    stale_flux<Z>(m, s, P, last, 4, false, tmp);
    for (int k = 0; k < 5; k++) s.s->fcarry[5 + k] = (double)tmp[k];
}

// Residual (4 faces + interphase sources, src/sr_source.F90:42-155) and the
// RK stage update of src/sr_RK.F90 fused; iblank == 1 cells.
// FACE: the four face fluxes are gathered from k_faceflux's output (face-
// based variants) instead of evaluated here.
template <bool ALIASED, bool FACE, int Z, bool ACC = false, bool NC = true>
__device__ __forceinline__ void k_flux_body(DevMesh m, DevState<R> s, DevParams P, int stage, int bid) {
    int i = bid * blockDim.x + threadIdx.x;
    if (i >= m.neles) return;
    if (ldg(m.iblank + i) != 1) return;
    // cells of the FP64 wall layers: updated by the FP64 kernels
    if (sizeof(R) != sizeof(double) && m.nwall > 0 && ldg(m.wclass + i)) return;
    double rhs[10];
#pragma unroll
    for (int k = 0; k < 10; k++) rhs[k] = 0.0;
    R Fg[5] = {R(0), R(0), R(0), R(0), R(0)}, Fp[5] = {R(0), R(0), R(0), R(0), R(0)};
    bool haveg = false, havep = false;
    if constexpr (ACC) {
        // face modes 2 and 3: the face sums were accumulated per cell
#pragma unroll
        for (int k = 0; k < 10; k++) rhs[k] = COL(s.racc, k)[i];
    } else if constexpr (FACE) {
#pragma unroll
        for (int f = 0; f < 4; f++) {
            const int code = ldg(COL(m.cface, f) + i);
            const int fid = (code > 0 ? code : -code) - 1;
            const R sg = code > 0 ? R(1) : R(-1);
            R e[FACE_REC];
            load_frec<NC>(s.ff + (size_t)FACE_REC * (size_t)fid, e);
#pragma unroll
            for (int k = 0; k < 10; k++) e[k] = sg * e[k];
            if (e[10] != R(0)) {
                rhs[1] = rhs[1] + (double)e[1]; rhs[2] = rhs[2] + (double)e[2]; rhs[3] = rhs[3] + (double)e[3];
                rhs[6] = rhs[6] + (double)e[6]; rhs[7] = rhs[7] + (double)e[7]; rhs[8] = rhs[8] + (double)e[8];
            } else {
#pragma unroll
                for (int k = 0; k < 10; k++) rhs[k] = rhs[k] + (double)e[k];
            }
        }
    }
#pragma unroll 1
    for (int f = 0; f < 4 && !FACE && !ACC; f++) {
        FaceOut o;
        unsigned bad_ = 0;
        face_eval<0, Z>(m, s, P, i, f, o, bad_, s.pr);
        if (o.wall) {
            rhs[1] = rhs[1] + (double)o.w[0]; rhs[2] = rhs[2] + (double)o.w[1];
            rhs[3] = rhs[3] + (double)o.w[2]; rhs[6] = rhs[6] + (double)o.w[3];
            rhs[7] = rhs[7] + (double)o.w[4]; rhs[8] = rhs[8] + (double)o.w[5];
            continue;
        }
        if (o.takeg) {
            for (int k = 0; k < 5; k++) Fg[k] = o.F[k];
            haveg = true;
        } else if (ALIASED && !haveg) {
            stale_flux<Z>(m, s, P, i, f, true, Fg);
            haveg = true;
        }
        if (o.takep) {
            for (int k = 0; k < 5; k++) Fp[k] = o.F[5 + k];
            havep = true;
        } else if (ALIASED && !havep) {
            stale_flux<Z>(m, s, P, i, f, false, Fp);
            havep = true;
        }
#pragma unroll
        for (int k = 0; k < 5; k++) {
            rhs[k] = rhs[k] + (double)Fg[k];
            rhs[5 + k] = rhs[5 + k] + (double)Fp[k];
        }
    }
    // interphase sources with the 1/r-weighted LSQ gradient of alpha_g
    {
        const double* pr = s.pr;
        const R tg = (R)COL(pr, P_TG)[i], phig = (R)COL(pr, P_PHIG)[i], rog = (R)COL(pr, P_ROG)[i];
        const R rop = (R)COL(pr, P_ROP)[i], phip = (R)COL(pr, P_PHIP)[i];
        const R ug = (R)COL(pr, P_UG)[i], vg = (R)COL(pr, P_VG)[i], wg = (R)COL(pr, P_WG)[i];
        const R up = (R)COL(pr, P_UP)[i], vp = (R)COL(pr, P_VP)[i], wp = (R)COL(pr, P_WP)[i];
        const R tp = (R)COL(pr, P_TP)[i], pg = (R)COL(pr, P_PG)[i];
        const R dl = (R)ldg(m.dl + i), voli = (R)ldg(m.vol + i);
        const R amug = (R)P.as * sqrt(tg) / (R(1) + (R)P.ts / tg);
        const R du = ug - up, dv = vg - vp, dw = wg - wp;
        // alpha_g (alpha_g - 1) and 1 - alpha_g in the reference's form in
        // FP64; from alpha_p in FP32, where the differences would cancel
        // (see face_eval)
        // (with dispersed phases alpha_p is not 1 - alpha_g, which FP32 then
        // forms in FP64)
        R drag, omg;
        if constexpr (sizeof(R) == 4) {
            omg = P.five_phase ? (R)(1.0 - COL(s.pr, P_PHIG)[i]) : phip;
            drag = -(R(0.44) * phig * omg) * rog * sqrt(du * du + dv * dv + dw * dw) * dl;
        } else {
            omg = R(1) - phig;
            drag = R(0.44) * phig * (phig - R(1)) * rog * sqrt(du * du + dv * dv + dw * dw) * dl;
        }
        const R fdgx = drag * du, fdgy = drag * dv, fdgz = drag * dw;
        const R qsource = R(6) * phip * amug * (R)P.cpg * R(2) * (tp - tg) / ((R)P.prg * (dl * dl));
        const R delpstar = R(2) * (phig * rog * phip * rop) / (phig * rop + phip * rog) *
                           (du * du + dv * dv + dw * dw);
        const R pint = pg - mn2(delpstar, R(0.01) * pg);
        const R den = phig * rog + omg * rop;
        const R rden = rcp(den);
        const R uint_ = div_rn(phig * rog * ug + omg * rop * up, den, rden);
        const R vint = div_rn(phig * rog * vg + omg * rop * vp, den, rden);
        const R wint = div_rn(phig * rog * wg + omg * rop * wp, den, rden);
        const double x0 = ldg(m.xc + i), y0 = ldg(m.yc + i), z0 = ldg(m.zc + i);
        R xa[4], ya[4], za[4], pa[4], wt[4];
#pragma unroll
        for (int f = 0; f < 4; f++) {
            int n = ldg(COL(m.nc, f) + i);
            xa[f] = (R)(ldg(m.xc + n) - x0);
            ya[f] = (R)(ldg(m.yc + n) - y0);
            za[f] = (R)(ldg(m.zc + n) - z0);
            pa[f] = (R)(COL(pr, P_PHIG)[n] - COL(pr, P_PHIG)[i]);
        }
        R rw[4];
#if HP_LSQ_TABLE
#pragma unroll
        for (int f = 0; f < 4; f++) { wt[f] = (R)ldg(COL(m.lsqb, f) + i); rw[f] = rcp(wt[f]); }
        const R a1 = (R)ldg(COL(m.lsqb, 4) + i), a2 = (R)ldg(COL(m.lsqb, 5) + i), a3 = (R)ldg(COL(m.lsqb, 6) + i);
        const R b1 = (R)ldg(COL(m.lsqb, 7) + i), b2 = (R)ldg(COL(m.lsqb, 8) + i), b3 = (R)ldg(COL(m.lsqb, 9) + i);
#else
#pragma unroll
        for (int f = 0; f < 4; f++) { wt[f] = sqrt(xa[f] * xa[f] + ya[f] * ya[f] + za[f] * za[f]); rw[f] = rcp(wt[f]); }
        const R a1 = DW(xa[0] * xa[0], 0) + DW(xa[1] * xa[1], 1) + DW(xa[2] * xa[2], 2) + DW(xa[3] * xa[3], 3);
        const R a2 = DW(ya[0] * ya[0], 0) + DW(ya[1] * ya[1], 1) + DW(ya[2] * ya[2], 2) + DW(ya[3] * ya[3], 3);
        const R a3 = DW(za[0] * za[0], 0) + DW(za[1] * za[1], 1) + DW(za[2] * za[2], 2) + DW(za[3] * za[3], 3);
        const R b1 = DW(xa[0] * ya[0], 0) + DW(xa[1] * ya[1], 1) + DW(xa[2] * ya[2], 2) + DW(xa[3] * ya[3], 3);
        const R b2 = DW(xa[0] * za[0], 0) + DW(xa[1] * za[1], 1) + DW(xa[2] * za[2], 2) + DW(xa[3] * za[3], 3);
        const R b3 = DW(ya[0] * za[0], 0) + DW(ya[1] * za[1], 1) + DW(ya[2] * za[2], 2) + DW(ya[3] * za[3], 3);
#endif
        R c1 = DW(pa[0] * xa[0], 0) + DW(pa[1] * xa[1], 1) + DW(pa[2] * xa[2], 2) + DW(pa[3] * xa[3], 3);
        R c2 = DW(pa[0] * ya[0], 0) + DW(pa[1] * ya[1], 1) + DW(pa[2] * ya[2], 2) + DW(pa[3] * ya[3], 3);
        R c3 = DW(pa[0] * za[0], 0) + DW(pa[1] * za[1], 1) + DW(pa[2] * za[2], 2) + DW(pa[3] * za[3], 3);
#if HP_LSQ_TABLE
        const R dnr = (R)ldg(COL(m.lsqb, 10) + i);
#else
        const R dnr = det3(a1, b1, b2, b1, a2, b3, b2, b3, a3);
#endif
        const R rdnr = rcp(dnr);
        R dpx = div_rn(det3(c1, c2, c3, b1, a2, b3, b2, b3, a3), dnr, rdnr);
        R dpy = div_rn(det3(a1, b1, b2, c1, c2, c3, b2, b3, a3), dnr, rdnr);
        R dpz = div_rn(det3(a1, b1, b2, b1, a2, b3, c1, c2, c3), dnr, rdnr);
        const R g = R(0);   // gravity (src/main.F90:341)
        R en = pint * (uint_ * dpx + vint * dpy + wint * dpz) + uint_ * fdgx + vint * fdgy + wint * fdgz + qsource;
        const double* vis = s.vis;
        rhs[1] = rhs[1] - (double)((fdgx + pint * dpx + phig * rog * g) * voli) - COL(vis, 0)[i];
        rhs[2] = rhs[2] - (double)((fdgy + pint * dpy) * voli) - COL(vis, 1)[i];
        rhs[3] = rhs[3] - (double)((fdgz + pint * dpz) * voli) - COL(vis, 2)[i];
        rhs[4] = rhs[4] - (double)(en * voli) - COL(vis, 3)[i];
        rhs[6] = rhs[6] + (double)((fdgx + pint * dpx - phip * rop * g) * voli) - COL(vis, 4)[i];
        rhs[7] = rhs[7] + (double)((fdgy + pint * dpy) * voli) - COL(vis, 5)[i];
        rhs[8] = rhs[8] + (double)((fdgz + pint * dpz) * voli) - COL(vis, 6)[i];
        rhs[9] = rhs[9] + (double)(en * voli) - COL(vis, 7)[i];
    }
    // five-phase: drag of q, r, s on the liquid, in the order
    // src/sr_sourceqrs.F90 adds it
    if (P.five_phase) {
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
            for (int c = 0; c < 3; c++) rhs[6 + c] = rhs[6 + c] + COL(s.qdrag, 3 * d + c)[i];
    }
    // RK stage update (FP64)
    const double dtbyvol = s.s[case_of(m, i)].dt / ldg(m.vol + i);
#pragma unroll
    for (int j = 0; j < 10; j++) {
        const double r = rhs[j] - COL(s.d24, j)[i];
        const double cu = COL(s.cu, j)[i];
        double* cnp = COL(s.cn, j) + i;
        if (P.rk_scheme == 0) {
            if (stage == 1) {
                double v = cu - (11.0 / 20.0) * dtbyvol * r;
                *cnp = v;
                COL(s.cn1, j)[i] = v;
            } else {
                double upd = *cnp - (11.0 / 20.0) * dtbyvol * r;
                if (stage == 2) *cnp = (3.0 / 8.0) * cu + (5.0 / 8.0) * upd;
                else if (stage == 3) *cnp = (4.0 / 9.0) * cu + (5.0 / 9.0) * upd;
                else *cnp = (111.0 / 1331.0) * cu + (260.0 / 1331.0) * COL(s.cn1, j)[i] + (960.0 / 1331.0) * upd;
            }
        } else {
            if (stage == 1) *cnp = cu - dtbyvol * r;
            else {
                double upd = *cnp - dtbyvol * r;
                if (stage == 2) *cnp = 0.75 * cu + 0.25 * upd;
                else *cnp = (1.0 / 3.0) * cu + (2.0 / 3.0) * upd;
            }
        }
    }
}
template <bool ALIASED, bool FACE, int Z, bool ACC = false>
__global__ void __launch_bounds__(128) k_flux(DevMesh m, DevState<R> s, DevParams P, int stage) {
    k_flux_body<ALIASED, FACE, Z, ACC>(m, s, P, stage, blockIdx.x);
}


// ---------------------------------------------------------------------------
// Venkatakrishnan limiter of the four-lane gradient kernel: lane q limits
// pg, pp, rog or rop from the gradient it holds (lg) or receives (sg of
// another lane), over its four faces; lane 0 stores the cell's minimum.
// lp, lc (the staged kernel, below): the limiter field of the lane's cell
// and of its four neighbours (lp[k * LIM_LD], k = 0 the cell) and the cell's
// face centroids and epsilon^2 (lc[k * LIMC_LD], k = 0..11 fch, 12 eps2),
// copied to shared memory when the kernel started; null: read from global
// memory
__device__ __forceinline__ unsigned grad4_limiter(const DevMesh& m, const DevState<R>& s, const DevParams& P,
                                                  int i, int q, bool active, const int n[4], double x0,
                                                  double y0, double z0, R lg[3], const R sg[3],
                                                  const double* lp, const double* lc) {
    // lane 2 takes rog from lane 3, lane 3 takes rop from lane 0
    const int src = q == 2 ? 3 : (q == 3 ? 0 : q);
    R fx0 = qshfl(sg[0], src), fy0 = qshfl(sg[1], src), fz0 = qshfl(sg[2], src);
    if (q >= 2) { lg[0] = fx0; lg[1] = fy0; lg[2] = fz0; }
    const int lcol = q == 0 ? P_PG : q == 1 ? P_PP : q == 2 ? P_ROG : P_ROP;
    if (lp) {
        cp_async_wait_all();
        __syncwarp();
    }
    const R epssq = lc ? (R)lc[12 * LIMC_LD] : (R)ldg(m.eps2 + i);
    const R* qq = COL(s.prr, lcol);
    R qi = lp ? (R)lp[0] : qq[i];
    R q0 = lp ? (R)lp[LIM_LD] : qq[n[0]], q1 = lp ? (R)lp[2 * LIM_LD] : qq[n[1]];
    R q2 = lp ? (R)lp[3 * LIM_LD] : qq[n[2]], q3 = lp ? (R)lp[4 * LIM_LD] : qq[n[3]];
    R vmax = mx2(mx2(mx2(mx2(qi, q0), q1), q2), q3);
    R vmin = mn2(mn2(mn2(mn2(qi, q0), q1), q2), q3);
    R dmax = (R)(vmax - qi), dmin = (R)(vmin - qi);
    R phl = R(0);
#pragma unroll
    for (int f = 0; f < 4; f++) {
        R fx = (R)((lc ? lc[f * LIMC_LD] : ldg(COL(m.fch, f) + i)) - x0);
        R fy = (R)((lc ? lc[(4 + f) * LIMC_LD] : ldg(COL(m.fch, 4 + f) + i)) - y0);
        R fz = (R)((lc ? lc[(8 + f) * LIMC_LD] : ldg(COL(m.fch, 8 + f) + i)) - z0);
        R d = fx * lg[0] + fy * lg[1] + fz * lg[2];
        R ph;
        if (d > R(0)) ph = fvenkat(dmax, d, epssq);
        else if (d < R(0)) ph = fvenkat(dmin, d, epssq);
        else ph = R(1);
        phl = (f == 0) ? ph : mn2(phl, ph);
    }
    R p0 = qshfl(phl, 0), p1 = qshfl(phl, 1), p2 = qshfl(phl, 2), p3 = qshfl(phl, 3);
    if (q == 0 && active) s.phi[i] = (double)mn2(mn2(mn2(p0, p1), p2), p3);
    return 0u;
}

// Staged form of the four-lane gradient kernel (HP_GRAD4_STAGE, FP64
// variants with set-up tables): when a block starts, each lane issues
// asynchronous copies into shared memory of
//   group 0   the 28 geometry values of its cell (12 centroid differences,
//             the 16 LSQA terms), lane q copying values q, q + 4, ...;
//   groups 1-4  field q + 4r (r = 0..3) at the cell and its 4 neighbours
//             (an empty group when the lane has no such field);
//   group 5   the limiter's inputs (see grad4_limiter).
// The field loop waits for one group per field, so the gathers of later
// fields stay in flight while earlier ones are computed, without holding
// registers.
#ifndef HP_GRAD4_STAGE
#define HP_GRAD4_STAGE 0
#endif
#define GRAD4_STAGED (HP_GRAD4_STAGE && HP_DXN_TABLE && HP_LSQ_TABLE)
enum { GEO_N = 28, GEO_LD = 32 };
struct Grad4Stage {
    const double* geo;    // geo[k * GEO_LD], k < 12 centroid differences, 12 + j LSQA column j
    const double* gat;    // gat[(5 r + k) * LIM_LD], field q + 4r at the cell (k = 0) and neighbour k - 1
    const double* lim;    // see grad4_limiter
    const double* limc;
};

// ---------------------------------------------------------------------------
// k_grad with four lanes per cell: lane q computes the LSQ gradients of
// fields q, q+4, q+8, q+12 and the limiter of one of pg, pp, rog, rop; phi is
// the in-order minimum over the lanes (equal to the reference's chain when no
// value is NaN).  F selects the division form (see mdiv); the return value is
// the fast form's out-of-range flag.  st: the staged copies (null: read from
// global memory).
template <int F>
__device__ __forceinline__ unsigned grad4_body(const DevMesh& m, const DevState<R>& s, const DevParams& P, int i,
                                               int q, bool active, const Grad4Stage* st) {
    unsigned bad = 0;
    int n[4];
#pragma unroll
    for (int f = 0; f < 4; f++) n[f] = ldg(COL(m.nc, f) + i);
    const double x0 = ldg(m.xc + i), y0 = ldg(m.yc + i), z0 = ldg(m.zc + i);
#if GRAD4_STAGED
    if constexpr (sizeof(R) == sizeof(double)) {
        const double* geo = st->geo;
        cp_async_wait_group<5>();   // group 0, copied by the cell's four lanes
        __syncwarp();
#define GX(f) geo[(3 * (f)) * GEO_LD]
#define GY(f) geo[(3 * (f) + 1) * GEO_LD]
#define GZ(f) geo[(3 * (f) + 2) * GEO_LD]
#define GT(j) geo[(12 + (j)) * GEO_LD]
#undef DW
#define DW(x, f) mdiv<F>((x), GT(f), GT(11 + (f)), bad)
#pragma unroll
        for (int f = 0; f < 4; f++) (void)mrcp_tab<F>(GT(f), GT(11 + f), bad);
        (void)mrcp_tab<F>(GT(10), GT(15), bad);
        R lg[3] = {R(0), R(0), R(0)};
        R sg[3] = {R(0), R(0), R(0)};
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int v = q + 4 * r;
            if (v >= 13) break;
            if (r == 0) cp_async_wait_group<4>();
            else if (r == 1) cp_async_wait_group<3>();
            else if (r == 2) cp_async_wait_group<2>();
            else cp_async_wait_group<1>();
            const double* g = st->gat + 5 * r * LIM_LD;
            const R qi = (R)g[0];
            const R qa = (R)(g[LIM_LD] - qi), qb = (R)(g[2 * LIM_LD] - qi);
            const R qc = (R)(g[3 * LIM_LD] - qi), qd = (R)(g[4 * LIM_LD] - qi);
            R c1 = DW(qa * GX(0), 0) + DW(qb * GX(1), 1) + DW(qc * GX(2), 2) + DW(qd * GX(3), 3);
            R c2;
            if (v == 7)   // cTp2 lacks the /wt4 (src/sr_derivative.F90:225)
                c2 = DW(qa * GY(0), 0) + DW(qb * GY(1), 1) + DW(qc * GY(2), 2) + qd * GY(3);
            else
                c2 = DW(qa * GY(0), 0) + DW(qb * GY(1), 1) + DW(qc * GY(2), 2) + DW(qd * GY(3), 3);
            R c3 = DW(qa * GZ(0), 0) + DW(qb * GZ(1), 1) + DW(qc * GZ(2), 2) + DW(qd * GZ(3), 3);
            const R a1 = GT(4), a2 = GT(5), a3 = GT(6), b1 = GT(7), b2 = GT(8), b3 = GT(9);
            const R dnr = GT(10), rdnr = GT(15);
            R gx = mdiv<F>(det3(c1, c2, c3, b1, a2, b3, b2, b3, a3), dnr, rdnr, bad);
            R gy = mdiv<F>(det3(a1, b1, b2, c1, c2, c3, b2, b3, a3), dnr, rdnr, bad);
            R gz = mdiv<F>(det3(a1, b1, b2, b1, a2, b3, c1, c2, c3), dnr, rdnr, bad);
            if (v < 11 && active) {
                COL(s.gr, 3 * v + 0)[i] = gx;
                COL(s.gr, 3 * v + 1)[i] = gy;
                COL(s.gr, 3 * v + 2)[i] = gz;
            }
            if (v == 8 || v == 9) { lg[0] = gx; lg[1] = gy; lg[2] = gz; }
            if (v == 11 || v == 12) { sg[0] = gx; sg[1] = gy; sg[2] = gz; }
        }
#undef DW
#undef GX
#undef GY
#undef GZ
#undef GT
#define DW(x, f) div_rn((x), wt[f], rw[f])
        return bad | grad4_limiter(m, s, P, i, q, active, n, x0, y0, z0, lg, sg, st->lim, st->limc);
    }
#endif
    (void)st;
    R xa[4], ya[4], za[4];
#pragma unroll
    for (int f = 0; f < 4; f++) {
#if HP_DXN_TABLE
        // the centroid differences, formed at set-up (the same subtraction)
        xa[f] = (R)ldg(COL(m.dxn, 3 * f) + i);
        ya[f] = (R)ldg(COL(m.dxn, 3 * f + 1) + i);
        za[f] = (R)ldg(COL(m.dxn, 3 * f + 2) + i);
#else
        xa[f] = (R)(ldg(m.xc + n[f]) - x0);
        ya[f] = (R)(ldg(m.yc + n[f]) - y0);
        za[f] = (R)(ldg(m.zc + n[f]) - z0);
#endif
    }
    // geometry-only terms (wt, a1..b3, dnr of src/sr_derivative.F90:163-176,
    // 255), evaluated once at set-up with the same expressions
    R wt[4], rw[4];
#undef DW
#define DW(x, f) mdiv<F>((x), wt[f], rw[f], bad)
#if HP_LSQ_TABLE
#pragma unroll
    for (int f = 0; f < 4; f++) {
        wt[f] = (R)ldg(COL(m.lsqa, f) + i);
        rw[f] = mrcp_tab<F>(wt[f], (R)ldg(COL(m.lsqa, 11 + f) + i), bad);
    }
    const R a1 = (R)ldg(COL(m.lsqa, 4) + i), a2 = (R)ldg(COL(m.lsqa, 5) + i), a3 = (R)ldg(COL(m.lsqa, 6) + i);
    const R b1 = (R)ldg(COL(m.lsqa, 7) + i), b2 = (R)ldg(COL(m.lsqa, 8) + i), b3 = (R)ldg(COL(m.lsqa, 9) + i);
    const R dnr = (R)ldg(COL(m.lsqa, 10) + i);
    const R rdnr_tab = (R)ldg(COL(m.lsqa, 15) + i);
#else
#pragma unroll
    for (int f = 0; f < 4; f++) { wt[f] = xa[f] * xa[f] + ya[f] * ya[f] + za[f] * za[f]; rw[f] = mrcp<F>(wt[f], bad); }
    const R a1 = DW(xa[0] * xa[0], 0) + DW(xa[1] * xa[1], 1) + DW(xa[2] * xa[2], 2) + DW(xa[3] * xa[3], 3);
    const R a2 = DW(ya[0] * ya[0], 0) + DW(ya[1] * ya[1], 1) + DW(ya[2] * ya[2], 2) + DW(ya[3] * ya[3], 3);
    const R a3 = DW(za[0] * za[0], 0) + DW(za[1] * za[1], 1) + DW(za[2] * za[2], 2) + DW(za[3] * za[3], 3);
    const R b1 = DW(xa[0] * ya[0], 0) + DW(xa[1] * ya[1], 1) + DW(xa[2] * ya[2], 2) + DW(xa[3] * ya[3], 3);
    const R b2 = DW(xa[0] * za[0], 0) + DW(xa[1] * za[1], 1) + DW(xa[2] * za[2], 2) + DW(xa[3] * za[3], 3);
    const R b3 = DW(za[0] * ya[0], 0) + DW(za[1] * ya[1], 1) + DW(za[2] * ya[2], 2) + DW(za[3] * ya[3], 3);
    const R dnr = det3(a1, b1, b2, b1, a2, b3, b2, b3, a3);
#endif
#if HP_LSQ_TABLE
    const R rdnr = mrcp_tab<F>(dnr, rdnr_tab, bad);
#else
    const R rdnr = mrcp<F>(dnr, bad);
#endif
    const int pcol[13] = {P_UG, P_VG, P_WG, P_TG, P_UP, P_VP, P_WP, P_TP, P_PG, P_PP, P_PHIG, P_ROG, P_ROP};
    // limiter field of this lane: pg (grad field 8), pp (9), rog (11), rop (12)
    R lg[3] = {R(0), R(0), R(0)};     // gradient of the lane's limiter field
    R sg[3] = {R(0), R(0), R(0)};     // gradient this lane forwards to another lane
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int v = q + 4 * r;
        if (v >= 13) break;
        const R* qq = COL(s.prr, pcol[v]);
        R qi = qq[i];
        R qa = (R)(qq[n[0]] - qi), qb = (R)(qq[n[1]] - qi), qc = (R)(qq[n[2]] - qi), qd = (R)(qq[n[3]] - qi);
        R c1 = DW(qa * xa[0], 0) + DW(qb * xa[1], 1) + DW(qc * xa[2], 2) + DW(qd * xa[3], 3);
        R c2;
        if (v == 7)   // cTp2 lacks the /wt4 (src/sr_derivative.F90:225)
            c2 = DW(qa * ya[0], 0) + DW(qb * ya[1], 1) + DW(qc * ya[2], 2) + qd * ya[3];
        else
            c2 = DW(qa * ya[0], 0) + DW(qb * ya[1], 1) + DW(qc * ya[2], 2) + DW(qd * ya[3], 3);
        R c3 = DW(qa * za[0], 0) + DW(qb * za[1], 1) + DW(qc * za[2], 2) + DW(qd * za[3], 3);
        R gx = mdiv<F>(det3(c1, c2, c3, b1, a2, b3, b2, b3, a3), dnr, rdnr, bad);
        R gy = mdiv<F>(det3(a1, b1, b2, c1, c2, c3, b2, b3, a3), dnr, rdnr, bad);
        R gz = mdiv<F>(det3(a1, b1, b2, b1, a2, b3, c1, c2, c3), dnr, rdnr, bad);
        if (v < 11 && active) {
            COL(s.gr, 3 * v + 0)[i] = gx;
            COL(s.gr, 3 * v + 1)[i] = gy;
            COL(s.gr, 3 * v + 2)[i] = gz;
        }
        if (v == 8 || v == 9) { lg[0] = gx; lg[1] = gy; lg[2] = gz; }          // lanes 0, 1
        if (v == 11 || v == 12) { sg[0] = gx; sg[1] = gy; sg[2] = gz; }        // lanes 3, 0
    }
#undef DW
#define DW(x, f) div_rn((x), wt[f], rw[f])
    return bad | grad4_limiter(m, s, P, i, q, active, n, x0, y0, z0, lg, sg, nullptr, nullptr);
}


// LIST = 1: the cells of m.gcells (the FP64 wall layers and their
// neighbours) instead of all cells.
template <int LIST>
__device__ __forceinline__ void k_grad4_body(DevMesh m, DevState<R> s, DevParams P, int bid) {
    const long long gt = (long long)bid * blockDim.x + threadIdx.x;
    const int q = (int)(gt & 3);
    const int ncell = LIST ? m.ngwall : m.neles;
    const long long c = gt >> 2;
    const bool valid = c < ncell;
    const int k = valid ? (int)c : ncell - 1;
    const int i = LIST ? ldg(m.gcells + k) : k;
    const bool active = valid && grad_cell(ldg(m.iblank + i));
#if GRAD4_STAGED
    if constexpr (sizeof(R) == sizeof(double)) {
        __shared__ __align__(16) double sgeo[GEO_N * GEO_LD];
        __shared__ __align__(16) double sgat[4 * 5 * LIM_LD];
        __shared__ __align__(16) double slim[5 * LIM_LD];
        __shared__ __align__(16) double slimc[LIMC_N * LIMC_LD];
        const int tid = (int)threadIdx.x & (LIM_LD - 1), cl = (int)(threadIdx.x >> 2) & (GEO_LD - 1);
        int nn[4];
#pragma unroll
        for (int f = 0; f < 4; f++) nn[f] = ldg(COL(m.nc, f) + i);
        // group 0: geometry values q, q + 4, ... of the lane's cell
#pragma unroll
        for (int k = q; k < GEO_N; k += 4)
            cp_async8(sgeo + k * GEO_LD + cl, k < 12 ? COL(m.dxn, k) + i : COL(m.lsqa, k - 12) + i);
        cp_async_commit();
        // groups 1-4: fields q, q + 4, q + 8, q + 12
        const int pcol[13] = {P_UG, P_VG, P_WG, P_TG, P_UP, P_VP, P_WP, P_TP, P_PG, P_PP, P_PHIG, P_ROG, P_ROP};
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int v = q + 4 * r;
            if (v < 13) {
                const double* qv = reinterpret_cast<const double*>(COL(s.prr, pcol[v]));
                double* g = sgat + 5 * r * LIM_LD + tid;
                cp_async8(g, qv + i);
#pragma unroll
                for (int f = 0; f < 4; f++) cp_async8(g + (1 + f) * LIM_LD, qv + nn[f]);
            }
            cp_async_commit();
        }
        // group 5: the limiter field at the cell and its neighbours, face
        // centroid columns q, 4 + q, 8 + q and (lane 0) epsilon^2
        const int lcol = q == 0 ? P_PG : q == 1 ? P_PP : q == 2 ? P_ROG : P_ROP;
        const double* ql = reinterpret_cast<const double*>(COL(s.prr, lcol));
        cp_async8(slim + tid, ql + i);
#pragma unroll
        for (int f = 0; f < 4; f++) cp_async8(slim + (1 + f) * LIM_LD + tid, ql + nn[f]);
#pragma unroll
        for (int d = 0; d < 3; d++) cp_async8(slimc + (4 * d + q) * LIMC_LD + cl, COL(m.fch, 4 * d + q) + i);
        if (q == 0) cp_async8(slimc + 12 * LIMC_LD + cl, m.eps2 + i);
        cp_async_commit();
        const Grad4Stage st{sgeo + cl, sgat + tid, slim + tid, slimc + cl};
        if constexpr (HP_FAST(1)) {
            const unsigned bad = grad4_body<1>(m, s, P, i, q, active, &st);
            if (__any_sync(0xffffffffu, bad)) grad4_body<0>(m, s, P, i, q, active, &st);
        } else {
            grad4_body<0>(m, s, P, i, q, active, &st);
        }
        // the fused step reuses the arrays for its next virtual block
        __syncwarp();
        return;
    }
#endif
    if constexpr (HP_FAST(1)) {
        // the outputs are not inputs of this kernel, so a warp that flagged
        // an operand simply recomputes and overwrites them
        const unsigned bad = grad4_body<1>(m, s, P, i, q, active, nullptr);
        if (__any_sync(0xffffffffu, bad)) grad4_body<0>(m, s, P, i, q, active, nullptr);
    } else {
        grad4_body<0>(m, s, P, i, q, active, nullptr);
    }
}
template <int LIST>
__global__ void __launch_bounds__(128, HP_GRAD4_MINB) k_grad4(DevMesh m, DevState<R> s, DevParams P) {
    k_grad4_body<LIST>(m, s, P, blockIdx.x);
}

// Columns of the tail prefetch: dl, vol, the 16 LSQB terms, vis, d24, cu
// and cn; TAIL_LD cells (one 128-thread block) per column.  (Staging the 14
// primitives and the 12 centroid differences as well measured 2% slower:
// the face evaluation has just read the primitives.)
enum { TAIL_DL = 0, TAIL_VOL = 1, TAIL_LSQB = 2, TAIL_VIS = 18, TAIL_D24 = 26, TAIL_CU = 36, TAIL_CN = 46,
       TAIL_N = 56, TAIL_LD = 32 };
__device__ __forceinline__ const double* tail_col(const DevMesh& m, const DevState<R>& s, int k) {
    if (k == TAIL_DL) return m.dl;
    if (k == TAIL_VOL) return m.vol;
    if (k < TAIL_VIS) return m.lsqb + (size_t)(k - TAIL_LSQB) * m.ld;
    if (k < TAIL_D24) return s.vis + (size_t)(k - TAIL_VIS) * m.ld;
    if (k < TAIL_CU) return s.d24 + (size_t)(k - TAIL_D24) * m.ld;
    if (k < TAIL_CN) return s.cu + (size_t)(k - TAIL_CU) * m.ld;
    return s.cn + (size_t)(k - TAIL_CN) * m.ld;
}

// Residual + sources + RK update with four lanes per cell: lane q evaluates
// face q; every lane re-assembles the residual in face order and computes
// the sources; lane q writes variables q, q+4, q+8.  F selects the division
// form (see mdiv).  The fast form returns false, before any store, when a lane
// of the warp flagged an operand (cn is read and written here, so the stores
// must wait for that vote).
template <int F, int Z, bool NC = true, bool PF = false>
__device__ __forceinline__ bool flux4_body(const DevMesh& m, const DevState<R>& s, const DevParams& P, int stage,
                                           int i, int q, bool active, const double* pf = nullptr) {
    unsigned bad = 0;
    const R* pr = s.prr;
    // PF: the cell's own values after the face evaluation come from the
    // shared-memory copy that k_flux4_body started (pf[k * TAIL_LD], column
    // k of the TAIL_* map)
#define TL(k, expr) (PF ? (R)pf[(k) * TAIL_LD] : (R)(expr))
#define TLS(k, expr) (PF ? (S)pf[(k) * TAIL_LD] : (S)(expr))
    // this lane's face
    R eff[10];
    int flags;
    {
        FaceOut o;
        face_eval<F, Z, R, NC>(m, s, P, i, q, o, bad, s.prr);
        if (o.wall) {
#pragma unroll
            for (int k = 0; k < 10; k++) eff[k] = R(0);
            eff[1] = o.w[0]; eff[2] = o.w[1]; eff[3] = o.w[2];
            eff[6] = o.w[3]; eff[7] = o.w[4]; eff[8] = o.w[5];
        } else {
#pragma unroll
            for (int k = 0; k < 10; k++) eff[k] = o.F[k];
        }
        flags = (o.wall ? 1 : 0) | (o.takeg ? 2 : 0) | (o.takep ? 4 : 0);
    }
    if constexpr (PF) {
        cp_async_wait_all();
        __syncwarp();
    }
    // neighbour data for the alpha_g gradient of the sources
    const int nq = ldg(COL(m.nc, q) + i);
    const double x0 = ldg(m.xc + i), y0 = ldg(m.yc + i), z0 = ldg(m.zc + i);
#if HP_DXN_TABLE
    const R xq = (R)ldg(COL(m.dxn, 3 * q) + i), yq = (R)ldg(COL(m.dxn, 3 * q + 1) + i),
            zq = (R)ldg(COL(m.dxn, 3 * q + 2) + i);
#else
    const R xq = (R)(ldg(m.xc + nq) - x0), yq = (R)(ldg(m.yc + nq) - y0), zq = (R)(ldg(m.zc + nq) - z0);
#endif
    // alpha_g differences from the FP64 primitives (see k_grad)
    const R pq = (R)(COL(s.pr, P_PHIG)[nq] - COL(s.pr, P_PHIG)[i]);
    // residual in face order 1..4 (src/sr_hllcbatten.F90:534-552)
    S rhs[10];
#pragma unroll
    for (int k = 0; k < 10; k++) rhs[k] = S(0.0);
    R Fg[5] = {R(0), R(0), R(0), R(0), R(0)}, Fp[5] = {R(0), R(0), R(0), R(0), R(0)};
#pragma unroll
    for (int f = 0; f < 4; f++) {
        R e[10];
#pragma unroll
        for (int k = 0; k < 10; k++) e[k] = qshfl(eff[k], f);
        const int fl = qshfl(flags, f);
        if (fl & 1) {
            rhs[1] = rhs[1] + (S)e[1]; rhs[2] = rhs[2] + (S)e[2]; rhs[3] = rhs[3] + (S)e[3];
            rhs[6] = rhs[6] + (S)e[6]; rhs[7] = rhs[7] + (S)e[7]; rhs[8] = rhs[8] + (S)e[8];
        } else {
            if (fl & 2) {
#pragma unroll
                for (int k = 0; k < 5; k++) Fg[k] = e[k];
            }
            if (fl & 4) {
#pragma unroll
                for (int k = 0; k < 5; k++) Fp[k] = e[5 + k];
            }
#pragma unroll
            for (int k = 0; k < 5; k++) {
                rhs[k] = rhs[k] + (S)Fg[k];
                rhs[5 + k] = rhs[5 + k] + (S)Fp[k];
            }
        }
    }
    R xa[4], ya[4], za[4], pa[4];
#pragma unroll
    for (int f = 0; f < 4; f++) {
        xa[f] = qshfl(xq, f); ya[f] = qshfl(yq, f); za[f] = qshfl(zq, f); pa[f] = qshfl(pq, f);
    }
    // interphase sources (src/sr_source.F90:46-155)
    {
        const R tg = (R)COL(pr, P_TG)[i], phig = (R)COL(pr, P_PHIG)[i],
                rog = (R)COL(pr, P_ROG)[i];
        const R rop = (R)COL(pr, P_ROP)[i], phip = (R)COL(pr, P_PHIP)[i];
        const R ug = (R)COL(pr, P_UG)[i], vg = (R)COL(pr, P_VG)[i], wg = (R)COL(pr, P_WG)[i];
        const R up = (R)COL(pr, P_UP)[i], vp = (R)COL(pr, P_VP)[i], wp = (R)COL(pr, P_WP)[i];
        const R tp = (R)COL(pr, P_TP)[i], pg = (R)COL(pr, P_PG)[i];
        const R dl = TL(TAIL_DL, ldg(m.dl + i)), voli = TL(TAIL_VOL, ldg(m.vol + i));
        const R amug = (R)P.as * sqrt(tg) / (R(1) + (R)P.ts / tg);
        const R du = ug - up, dv = vg - vp, dw = wg - wp;
        // alpha_g (alpha_g - 1) and 1 - alpha_g in the reference's form in
        // FP64; from alpha_p in FP32, where the differences would cancel
        // (see face_eval)
        // (with dispersed phases alpha_p is not 1 - alpha_g, which FP32 then
        // forms in FP64)
        R drag, omg;
        if constexpr (sizeof(R) == 4) {
            omg = P.five_phase ? (R)(1.0 - COL(s.pr, P_PHIG)[i]) : phip;
            drag = -(R(0.44) * phig * omg) * rog * sqrt(du * du + dv * dv + dw * dw) * dl;
        } else {
            omg = R(1) - phig;
            drag = R(0.44) * phig * (phig - R(1)) * rog * sqrt(du * du + dv * dv + dw * dw) * dl;
        }
        const R fdgx = drag * du, fdgy = drag * dv, fdgz = drag * dw;
        const R qsource = R(6) * phip * amug * (R)P.cpg * R(2) * (tp - tg) / ((R)P.prg * (dl * dl));
        const R delpstar = R(2) * (phig * rog * phip * rop) / (phig * rop + phip * rog) *
                           (du * du + dv * dv + dw * dw);
        const R pint = pg - mn2(delpstar, R(0.01) * pg);
        const R den = phig * rog + omg * rop;
        // lane q < 3 evaluates component q of the interface velocity, of the
        // right-hand side of the alpha_g LSQ system and of its solution; the
        // results are exchanged with shuffles
        const R gq = q == 0 ? ug : (q == 1 ? vg : wg);
        const R pq_ = q == 0 ? up : (q == 1 ? vp : wp);
        const R vq_int = (phig * rog * gq + omg * rop * pq_) / den;
        const R uint_ = qshfl(vq_int, 0), vint = qshfl(vq_int, 1), wint = qshfl(vq_int, 2);
        // geometry-only terms (src/sr_source.F90:100-117), evaluated at set-up
        R wt[4], rw[4];
#undef DW
#define DW(x, f) mdiv<F>((x), wt[f], rw[f], bad)
#if HP_LSQ_TABLE
#define LB(k) TL(TAIL_LSQB + (k), ldg(COL(m.lsqb, k) + i))
#pragma unroll
        for (int f = 0; f < 4; f++) {
            wt[f] = LB(f);
            rw[f] = mrcp_tab<F>(wt[f], LB(11 + f), bad);
        }
        const R a1 = LB(4), a2 = LB(5), a3 = LB(6);
        const R b1 = LB(7), b2 = LB(8), b3 = LB(9);
#else
#pragma unroll
        for (int f = 0; f < 4; f++) { wt[f] = sqrt(xa[f] * xa[f] + ya[f] * ya[f] + za[f] * za[f]); rw[f] = mrcp<F>(wt[f], bad); }
        const R a1 = DW(xa[0] * xa[0], 0) + DW(xa[1] * xa[1], 1) + DW(xa[2] * xa[2], 2) + DW(xa[3] * xa[3], 3);
        const R a2 = DW(ya[0] * ya[0], 0) + DW(ya[1] * ya[1], 1) + DW(ya[2] * ya[2], 2) + DW(ya[3] * ya[3], 3);
        const R a3 = DW(za[0] * za[0], 0) + DW(za[1] * za[1], 1) + DW(za[2] * za[2], 2) + DW(za[3] * za[3], 3);
        const R b1 = DW(xa[0] * ya[0], 0) + DW(xa[1] * ya[1], 1) + DW(xa[2] * ya[2], 2) + DW(xa[3] * ya[3], 3);
        const R b2 = DW(xa[0] * za[0], 0) + DW(xa[1] * za[1], 1) + DW(xa[2] * za[2], 2) + DW(xa[3] * za[3], 3);
        const R b3 = DW(ya[0] * za[0], 0) + DW(ya[1] * za[1], 1) + DW(ya[2] * za[2], 2) + DW(ya[3] * za[3], 3);
#endif
#if HP_LSQ_TABLE
        const R dnr = LB(10);
#else
        const R dnr = det3(a1, b1, b2, b1, a2, b3, b2, b3, a3);
#endif
        R dir[4];
#pragma unroll
        for (int f = 0; f < 4; f++) dir[f] = q == 0 ? xa[f] : (q == 1 ? ya[f] : za[f]);
        const R cq = DW(pa[0] * dir[0], 0) + DW(pa[1] * dir[1], 1) + DW(pa[2] * dir[2], 2) + DW(pa[3] * dir[3], 3);
        const R c1 = qshfl(cq, 0), c2 = qshfl(cq, 1), c3 = qshfl(cq, 2);
        // Cramer: lane 0 replaces the first column by c, lane 1 the second,
        // lane 2 the third
        const R A11 = q == 0 ? c1 : a1, A21 = q == 0 ? c2 : b1, A31 = q == 0 ? c3 : b2;
        const R A12 = q == 1 ? c1 : b1, A22 = q == 1 ? c2 : a2, A32 = q == 1 ? c3 : b3;
        const R A13 = q >= 2 ? c1 : b2, A23 = q >= 2 ? c2 : b3, A33 = q >= 2 ? c3 : a3;
#if HP_LSQ_TABLE
        const R rdnr = mrcp_tab<F>(dnr, LB(15), bad);
#undef LB
        const R dq = mdiv<F>(det3(A11, A21, A31, A12, A22, A32, A13, A23, A33), dnr, rdnr, bad);
#else
        const R dq = det3(A11, A21, A31, A12, A22, A32, A13, A23, A33) / dnr;
#endif
        const R dpx = qshfl(dq, 0), dpy = qshfl(dq, 1), dpz = qshfl(dq, 2);
#undef DW
#define DW(x, f) div_rn((x), wt[f], rw[f])
        const R g = R(0);
        R en = pint * (uint_ * dpx + vint * dpy + wint * dpz) + uint_ * fdgx + vint * fdgy + wint * fdgz + qsource;
        const double* vis = s.vis;
        rhs[1] = rhs[1] - (S)((fdgx + pint * dpx + phig * rog * g) * voli) - TLS(TAIL_VIS + 0, COL(vis, 0)[i]);
        rhs[2] = rhs[2] - (S)((fdgy + pint * dpy) * voli) - TLS(TAIL_VIS + 1, COL(vis, 1)[i]);
        rhs[3] = rhs[3] - (S)((fdgz + pint * dpz) * voli) - TLS(TAIL_VIS + 2, COL(vis, 2)[i]);
        rhs[4] = rhs[4] - (S)(en * voli) - TLS(TAIL_VIS + 3, COL(vis, 3)[i]);
        rhs[6] = rhs[6] + (S)((fdgx + pint * dpx - phip * rop * g) * voli) - TLS(TAIL_VIS + 4, COL(vis, 4)[i]);
        rhs[7] = rhs[7] + (S)((fdgy + pint * dpy) * voli) - TLS(TAIL_VIS + 5, COL(vis, 5)[i]);
        rhs[8] = rhs[8] + (S)((fdgz + pint * dpz) * voli) - TLS(TAIL_VIS + 6, COL(vis, 6)[i]);
        rhs[9] = rhs[9] + (S)(en * voli) - TLS(TAIL_VIS + 7, COL(vis, 7)[i]);
    }
    // five-phase: drag of q, r, s on the liquid (see k_flux)
    if (P.five_phase) {
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
            for (int c = 0; c < 3; c++) rhs[6 + c] = rhs[6 + c] + (S)COL(s.qdrag, 3 * d + c)[i];
    }
    if constexpr (F == 1) {
        if (__any_sync(0xffffffffu, bad)) return false;
    }
    if (!active) return true;
    const S dtbyvol = (S)s.s[case_of(m, i)].dt / TLS(TAIL_VOL, ldg(m.vol + i));
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const int j = q + 4 * r;
        if (j >= 10) break;
        const S rr = rhs[j] - TLS(TAIL_D24 + j, COL(s.d24, j)[i]);
        const S cu = TLS(TAIL_CU + j, COL(s.cu, j)[i]);
        double* cnp = COL(s.cn, j) + i;
        if (P.rk_scheme == 0) {
            if (stage == 1) {
                S v = cu - S(11.0 / 20.0) * dtbyvol * rr;
                *cnp = v;
                COL(s.cn1, j)[i] = v;
            } else {
                S upd = TLS(TAIL_CN + j, *cnp) - S(11.0 / 20.0) * dtbyvol * rr;
                if (stage == 2) *cnp = S(3.0 / 8.0) * cu + S(5.0 / 8.0) * upd;
                else if (stage == 3) *cnp = S(4.0 / 9.0) * cu + S(5.0 / 9.0) * upd;
                else *cnp = S(111.0 / 1331.0) * cu + S(260.0 / 1331.0) * (S)COL(s.cn1, j)[i] + S(960.0 / 1331.0) * upd;
            }
        } else {
            if (stage == 1) *cnp = cu - dtbyvol * rr;
            else {
                S upd = TLS(TAIL_CN + j, *cnp) - dtbyvol * rr;
                if (stage == 2) *cnp = S(0.75) * cu + S(0.25) * upd;
                else *cnp = S(1.0 / 3.0) * cu + S(2.0 / 3.0) * upd;
            }
        }
    }
#undef TL
#undef TLS
    return true;
}

// LIST = 1: the cells of m.wcells (the FP64 wall layers) instead of all
// cells.  The FP32 variants leave the cells of the wall layers (wclass) to
// those FP64 kernels.
template <int Z, int LIST, bool NC = true>
__device__ __forceinline__ void k_flux4_body(DevMesh m, DevState<R> s, DevParams P, int stage, int bid) {
    const long long gt = (long long)bid * blockDim.x + threadIdx.x;
    const int q = (int)(gt & 3);
    const int ncell = LIST ? m.nwall : m.neles;
    const long long c = gt >> 2;
    const bool valid = c < ncell;
    const int k = valid ? (int)c : ncell - 1;
    const int i = LIST ? ldg(m.wcells + k) : k;
    bool active = valid && ldg(m.iblank + i) == 1;
    if (sizeof(R) != sizeof(double) && m.nwall > 0) active = active && !ldg(m.wclass + i);
#if HP_FLUX4_PREFETCH && HP_LSQ_TABLE && HP_DXN_TABLE
    if constexpr (NC && sizeof(R) == sizeof(double)) {
        // start the asynchronous copy of the values that the sources and the
        // RK update read (TAIL_*) while the faces are evaluated: for all
        // cells, the warp's 8 consecutive cells, 64 bytes per column; for a
        // cell list, lane q copies columns q, q + 4, ... of its own cell
        __shared__ __align__(16) double stail[TAIL_N * TAIL_LD];
        if constexpr (LIST == 0) {
            const int lane = (int)(threadIdx.x & 31), w8 = (int)((threadIdx.x >> 5) * 8);
            const long long c0 = ((long long)bid * blockDim.x + (threadIdx.x & ~31u)) >> 2;
            for (int t = lane; t < TAIL_N * 4; t += 32) {
                const int k = t >> 2, part = t & 3;
                cp_async16(stail + k * TAIL_LD + w8 + 2 * part, tail_col(m, s, k) + c0 + 2 * part);
            }
        } else {
            const int cs = (int)(threadIdx.x >> 2) & (TAIL_LD - 1);
            for (int k = q; k < TAIL_N; k += 4) cp_async8(stail + k * TAIL_LD + cs, tail_col(m, s, k) + i);
        }
        cp_async_commit();
        const double* pf = stail + ((threadIdx.x >> 2) & (TAIL_LD - 1));
        if constexpr (HP_FAST(2)) {
            if (!flux4_body<1, Z, NC, true>(m, s, P, stage, i, q, active, pf))
                flux4_body<0, Z, NC, true>(m, s, P, stage, i, q, active, pf);
        } else {
            flux4_body<0, Z, NC, true>(m, s, P, stage, i, q, active, pf);
        }
        return;
    }
#endif
    if constexpr (HP_FAST(2)) {
        if (!flux4_body<1, Z, NC>(m, s, P, stage, i, q, active)) flux4_body<0, Z, NC>(m, s, P, stage, i, q, active);
    } else {
        flux4_body<0, Z, NC>(m, s, P, stage, i, q, active);
    }
}
template <int Z, int LIST>
__global__ void __launch_bounds__(128, HP_FLUX4_MINB) k_flux4(DevMesh m, DevState<R> s, DevParams P, int stage) {
    k_flux4_body<Z, LIST>(m, s, P, stage, blockIdx.x);
}

// Face-based fluxes (FP32-arithmetic variants on meshes without aliased
// ghosts): every face is evaluated once, in its owner cell's orientation,
// instead of once from each side.  Phases with no HLLC branch taken (only
// with NaN states) contribute zero here.
template <int Z, bool NC = true>
__device__ __forceinline__ void k_faceflux_body(DevMesh m, DevState<R> s, DevParams P, int bid) {
    const int t = bid * blockDim.x + threadIdx.x;
    if (t >= m.nface) return;
    const int i = ldg(m.f_i + t), f = ldg(m.f_code + t) & 3;
    if (wall_face(m, i, f)) return;
    FaceOut o{};
    unsigned bad = 0;
    face_eval<0, Z, R, NC>(m, s, P, i, f, o, bad, s.prr);
    R rec[FACE_REC];
    if (o.wall) {
#pragma unroll
        for (int k = 0; k < 10; k++) rec[k] = R(0);
        rec[1] = o.w[0]; rec[2] = o.w[1]; rec[3] = o.w[2];
        rec[6] = o.w[3]; rec[7] = o.w[4]; rec[8] = o.w[5];
    } else {
#pragma unroll
        for (int k = 0; k < 10; k++) rec[k] = o.F[k];
    }
    rec[10] = o.wall ? R(1) : R(0);
    rec[11] = R(0);
    store_frec(s.ff + (size_t)FACE_REC * (size_t)t, rec);
}
template <int Z>
__global__ void __launch_bounds__(128, HP_FLUX4_MINB) k_faceflux(DevMesh m, DevState<R> s, DevParams P) {
    k_faceflux_body<Z>(m, s, P, blockIdx.x);
}

// Face modes 2 and 3: each face evaluated once, its flux added to the owner's
// accumulator and subtracted from the other cell's (a ghost has none).
// ATOMIC = false: the faces fids[0, n) of one colour, which share no cell;
// ATOMIC = true: every face, with atomic adds (the order of the additions,
// and so the last bits of the sums, vary from run to run).
template <int Z, bool ATOMIC>
__device__ __forceinline__ void k_facescatter_body(DevMesh m, DevState<R> s, DevParams P,
                                                                     const int* fids, int n, int bid) {
    const int t = bid * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int fid = ATOMIC ? t : ldg(fids + t);
    const int i = ldg(m.f_i + fid), f = ldg(m.f_code + fid) & 3;
    const int j = ldg(COL(m.nc, f) + i);
    FaceOut o{};
    unsigned bad = 0;
    face_eval<0, Z>(m, s, P, i, f, o, bad, s.prr);
    double e[10];
    if (o.wall) {
#pragma unroll
        for (int k = 0; k < 10; k++) e[k] = 0.0;
        e[1] = o.w[0]; e[2] = o.w[1]; e[3] = o.w[2];
        e[6] = o.w[3]; e[7] = o.w[4]; e[8] = o.w[5];
    } else {
#pragma unroll
        for (int k = 0; k < 10; k++) e[k] = (double)o.F[k];
    }
    const bool other = j < m.neles;
#pragma unroll
    for (int k = 0; k < 10; k++) {
        double* acc = COL(s.racc, k);
        if (ATOMIC) {
            atomicAdd(acc + i, e[k]);
            if (other) atomicAdd(acc + j, -e[k]);
        } else {
            acc[i] = acc[i] + e[k];
            if (other) acc[j] = acc[j] - e[k];
        }
    }
}
template <int Z, bool ATOMIC>
__global__ void __launch_bounds__(128, HP_FLUX4_MINB) k_facescatter(DevMesh m, DevState<R> s, DevParams P,
                                                                     const int* fids, int n) {
    k_facescatter_body<Z, ATOMIC>(m, s, P, fids, n, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Face-centred viscous fluxes, src/sr_viscousgp.F90:488-1138 (AMUP constant).
// One face f of cell i: face-centred LSQ over 5 (boundary) or 8 (interior)
// cell centres, Newtonian stresses and heat flux; c[8] = the face's
// contribution to visug..vistp.
template <int F, class PT>
__device__ __forceinline__ void visc_face(const DevMesh& m, const DevState<R>& s, const DevParams& P,
                                          int i, int f, const int nci[4], double c[8], unsigned& bad,
                                          const PT* pr) {
    const int fcol[8] = {P_UG, P_VG, P_WG, P_TG, P_UP, P_VP, P_WP, P_TP};
    const R c23 = (R)P.c23;
    const R scx = (R)ldg(COL(m.sc, 3 * f) + i), scy = (R)ldg(COL(m.sc, 3 * f + 1) + i),
            scz = (R)ldg(COL(m.sc, 3 * f + 2) + i);
    const double xf = ldg(COL(m.fcv, f) + i), yf = ldg(COL(m.fcv, 4 + f) + i),
                 zf = ldg(COL(m.fcv, 8 + f) + i);
    const int neigh = nci[f];
    R ff[8];
#pragma unroll
    for (int v = 0; v < 8; v++) ff[v] = (R)((COL(pr, fcol[v])[i] + COL(pr, fcol[v])[neigh]) * 0.5);
    const R phigf = (R)((COL(pr, P_PHIG)[i] + COL(pr, P_PHIG)[neigh]) * 0.5);
    const R phipf = (R)((COL(pr, P_PHIP)[i] + COL(pr, P_PHIP)[neigh]) * 0.5);
    const R tgf = ff[3];
    const R amug = (R)P.as * sqrt(tgf) / (R(1) + (R)P.ts / tgf);
    const R akg = mdiv<F>(amug * (R)P.cpg, (R)P.prg, (R)P.r_prg, bad);
    const R amup = (R)P.amup;
    const R akp = mdiv<F>(amup * (R)P.cpp, (R)P.prp, (R)P.r_prp, bad);
    int mm[8];
    int nm;
    mm[0] = nci[0]; mm[1] = nci[1]; mm[2] = nci[2]; mm[3] = nci[3];
    if (neigh >= m.neles) {
        mm[4] = i; nm = 5;
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) mm[4 + k] = ldg(COL(m.nc, k) + neigh);
        nm = 8;
    }
    R dx[8], dy[8], dz[8];
    for (int k = 0; k < nm; k++) {
        dx[k] = (R)(ldg(m.xc + mm[k]) - xf);
        dy[k] = (R)(ldg(m.yc + mm[k]) - yf);
        dz[k] = (R)(ldg(m.zc + mm[k]) - zf);
    }
    R a11 = dx[0] * dx[0], a22 = dy[0] * dy[0], a33 = dz[0] * dz[0];
    R a12 = dx[0] * dy[0], a13 = dx[0] * dz[0], a23 = dy[0] * dz[0];
    for (int k = 1; k < nm; k++) {
        a11 = a11 + dx[k] * dx[k]; a22 = a22 + dy[k] * dy[k]; a33 = a33 + dz[k] * dz[k];
        a12 = a12 + dx[k] * dy[k]; a13 = a13 + dx[k] * dz[k]; a23 = a23 + dy[k] * dz[k];
    }
    const R dnr = det3(a11, a12, a13, a12, a22, a23, a13, a23, a33);
    const R rdnr = mrcp<F>(dnr, bad);
    R gr[8][3];
#pragma unroll
    for (int v = 0; v < 8; v++) {
        const PT* q = COL(pr, fcol[v]);
        R d0 = (R)q[mm[0]] - ff[v];
        R b1 = d0 * dx[0], b2 = d0 * dy[0], b3 = d0 * dz[0];
        for (int k = 1; k < nm; k++) {
            R dk = (R)q[mm[k]] - ff[v];
            b1 = b1 + dk * dx[k]; b2 = b2 + dk * dy[k]; b3 = b3 + dk * dz[k];
        }
        gr[v][0] = mdiv<F>(det3(b1, b2, b3, a12, a22, a23, a13, a23, a33), dnr, rdnr, bad);
        gr[v][1] = mdiv<F>(det3(a11, a12, a13, b1, b2, b3, a13, a23, a33), dnr, rdnr, bad);
        gr[v][2] = mdiv<F>(det3(a11, a12, a13, a12, a22, a23, b1, b2, b3), dnr, rdnr, bad);
    }
    const R ugf = ff[0], vgf = ff[1], wgf = ff[2], upf = ff[4], vpf = ff[5], wpf = ff[6];
    R delvg = gr[0][0] + gr[1][1] + gr[2][2];
    R txxg = amug * (R(2) * gr[0][0] - c23 * delvg);
    R tyyg = amug * (R(2) * gr[1][1] - c23 * delvg);
    R tzzg = amug * (R(2) * gr[2][2] - c23 * delvg);
    R txyg = amug * (gr[1][0] + gr[0][1]);
    R txzg = amug * (gr[2][0] + gr[0][2]);
    R tyzg = amug * (gr[1][2] + gr[2][1]);
    R qxxg = ugf * txxg + vgf * txyg + wgf * txzg + akg * gr[3][0];
    R qyyg = ugf * txyg + vgf * tyyg + wgf * tyzg + akg * gr[3][1];
    R qzzg = ugf * txzg + vgf * tyzg + wgf * tzzg + akg * gr[3][2];
    R delvp = gr[4][0] + gr[5][1] + gr[6][2];
    R txxp = amup * (R(2) * gr[4][0] - c23 * delvp);
    R tyyp = amup * (R(2) * gr[5][1] - c23 * delvp);
    R tzzp = amup * (R(2) * gr[6][2] - c23 * delvp);
    R txyp = amup * (gr[5][0] + gr[4][1]);
    R txzp = amup * (gr[6][0] + gr[4][2]);
    R tyzp = amup * (gr[5][2] + gr[6][1]);
    R qxxp = upf * txxp + vpf * txyp + wpf * txzp + akp * gr[7][0];
    R qyyp = upf * txyp + vpf * tyyp + wpf * tyzp + akp * gr[7][1];
    R qzzp = upf * txzp + vpf * tyzp + wpf * tzzp + akp * gr[7][2];
    c[0] = (double)(phigf * (txxg * scx + txyg * scy + txzg * scz));
    c[1] = (double)(phigf * (txyg * scx + tyyg * scy + tyzg * scz));
    c[2] = (double)(phigf * (txzg * scx + tyzg * scy + tzzg * scz));
    c[3] = (double)(phigf * (qxxg * scx + qyyg * scy + qzzg * scz));
    c[4] = (double)(phipf * (txxp * scx + txyp * scy + txzp * scz));
    c[5] = (double)(phipf * (txyp * scx + tyyp * scy + tyzp * scz));
    c[6] = (double)(phipf * (txzp * scx + tyzp * scy + tzzp * scz));
    c[7] = (double)(phipf * (qxxp * scx + qyyp * scy + qzzp * scz));
}

// One phase of visc_face: the four contributions c[0..3] of phase ph
// (0 gas: visug, visvg, viswg, vistg; 1 liquid: visup..vistp) of face f of
// cell i, every value formed by the same operations in the same order as in
// visc_face.  The stencil loop runs over the points outermost, so the point
// offsets are not kept across the fields: every sum still adds its terms in
// point order 1..nm, starting from the first term.
#ifndef HP_VISC8_MINB
#define HP_VISC8_MINB 5
#endif
template <int F, class PT>
__device__ __forceinline__ void visc_face_ph(const DevMesh& m, const DevState<R>& s, const DevParams& P,
                                             int i, int f, const int nci[4], int ph, double c[4], unsigned& bad,
                                             const PT* pr) {
    const int c0 = ph ? P_UP : P_UG;          // u, v, w, T columns of the phase: c0 .. c0 + 3
    const R c23 = (R)P.c23;
    const R scx = (R)ldg(COL(m.sc, 3 * f) + i), scy = (R)ldg(COL(m.sc, 3 * f + 1) + i),
            scz = (R)ldg(COL(m.sc, 3 * f + 2) + i);
    const double xf = ldg(COL(m.fcv, f) + i), yf = ldg(COL(m.fcv, 4 + f) + i),
                 zf = ldg(COL(m.fcv, 8 + f) + i);
    const int neigh = nci[f];
    R ff[4];
#pragma unroll
    for (int v = 0; v < 4; v++) ff[v] = (R)((COL(pr, c0 + v)[i] + COL(pr, c0 + v)[neigh]) * 0.5);
    const R phif = (R)((COL(pr, P_PHIG + ph)[i] + COL(pr, P_PHIG + ph)[neigh]) * 0.5);
    R amu, ak;
    if (ph == 0) {
        const R tgf = ff[3];
        amu = (R)P.as * sqrt(tgf) / (R(1) + (R)P.ts / tgf);
        ak = mdiv<F>(amu * (R)P.cpg, (R)P.prg, (R)P.r_prg, bad);
    } else {
        amu = (R)P.amup;
        ak = mdiv<F>(amu * (R)P.cpp, (R)P.prp, (R)P.r_prp, bad);
    }
    const bool bnd = neigh >= m.neles;        // 5-point stencil: the cell's 4 neighbours and the cell
    R a11, a22, a33, a12, a13, a23, b[4][3];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        if (k >= 5 && bnd) break;
        const int mk = k < 4 ? nci[k] : (bnd ? i : ldg(COL(m.nc, k - 4) + neigh));
        const R dx = (R)(ldg(m.xc + mk) - xf), dy = (R)(ldg(m.yc + mk) - yf), dz = (R)(ldg(m.zc + mk) - zf);
        if (k == 0) {
            a11 = dx * dx; a22 = dy * dy; a33 = dz * dz; a12 = dx * dy; a13 = dx * dz; a23 = dy * dz;
        } else {
            a11 = a11 + dx * dx; a22 = a22 + dy * dy; a33 = a33 + dz * dz;
            a12 = a12 + dx * dy; a13 = a13 + dx * dz; a23 = a23 + dy * dz;
        }
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const R d = (R)COL(pr, c0 + v)[mk] - ff[v];
            if (k == 0) {
                b[v][0] = d * dx; b[v][1] = d * dy; b[v][2] = d * dz;
            } else {
                b[v][0] = b[v][0] + d * dx; b[v][1] = b[v][1] + d * dy; b[v][2] = b[v][2] + d * dz;
            }
        }
    }
    const R dnr = det3(a11, a12, a13, a12, a22, a23, a13, a23, a33);
    const R rdnr = mrcp<F>(dnr, bad);
    R gr[4][3];
#pragma unroll
    for (int v = 0; v < 4; v++) {
        gr[v][0] = mdiv<F>(det3(b[v][0], b[v][1], b[v][2], a12, a22, a23, a13, a23, a33), dnr, rdnr, bad);
        gr[v][1] = mdiv<F>(det3(a11, a12, a13, b[v][0], b[v][1], b[v][2], a13, a23, a33), dnr, rdnr, bad);
        gr[v][2] = mdiv<F>(det3(a11, a12, a13, a12, a22, a23, b[v][0], b[v][1], b[v][2]), dnr, rdnr, bad);
    }
    const R uf = ff[0], vf = ff[1], wf = ff[2];
    R delv = gr[0][0] + gr[1][1] + gr[2][2];
    R txx = amu * (R(2) * gr[0][0] - c23 * delv);
    R tyy = amu * (R(2) * gr[1][1] - c23 * delv);
    R tzz = amu * (R(2) * gr[2][2] - c23 * delv);
    R txy = amu * (gr[1][0] + gr[0][1]);
    R txz = amu * (gr[2][0] + gr[0][2]);
    R tyz = amu * (gr[1][2] + gr[2][1]);
    R qxx = uf * txx + vf * txy + wf * txz + ak * gr[3][0];
    R qyy = uf * txy + vf * tyy + wf * tyz + ak * gr[3][1];
    R qzz = uf * txz + vf * tyz + wf * tzz + ak * gr[3][2];
    c[0] = (double)(phif * (txx * scx + txy * scy + txz * scz));
    c[1] = (double)(phif * (txy * scx + tyy * scy + tyz * scz));
    c[2] = (double)(phif * (txz * scx + tyz * scy + tzz * scz));
    c[3] = (double)(phif * (qxx * scx + qyy * scy + qzz * scz));
}

// one thread per cell (aliased meshes)
__global__ void __launch_bounds__(128) k_visc(DevMesh m, DevState<R> s, DevParams P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.neles) return;
    if (ldg(m.iblank + i) != 1) return;
    double acc[8];
#pragma unroll
    for (int k = 0; k < 8; k++) acc[k] = 0.0;
    int nci[4];
#pragma unroll
    for (int f = 0; f < 4; f++) nci[f] = ldg(COL(m.nc, f) + i);
#pragma unroll 1
    for (int f = 0; f < 4; f++) {
        double c[8];
        unsigned bad_ = 0;
        visc_face<0>(m, s, P, i, f, nci, c, bad_, s.pr);
#pragma unroll
        for (int k = 0; k < 8; k++) acc[k] = acc[k] + c[k];
    }
#pragma unroll
    for (int k = 0; k < 8; k++) COL(s.vis, k)[i] = acc[k];
}

// ---------------------------------------------------------------------------
// Four lanes per cell (lane q = thread & 3 owns face q / field group q).
// Per-cell sums are re-assembled in face order 1..4 with warp shuffles, so
// the result is identical to the one-thread-per-cell kernels.  All 32 lanes
// of a warp reach every shuffle (out-of-range lanes replay the last cell and
// do not write).

__device__ __forceinline__ void k_visc4_body(DevMesh m, DevState<R> s, DevParams P, int bid) {
    const long long gt = (long long)bid * blockDim.x + threadIdx.x;
    const int q = (int)(gt & 3);
    int i = (int)(gt >> 2);
    const bool valid = i < m.neles;
    if (!valid) i = m.neles - 1;
    const bool active = valid && ldg(m.iblank + i) == 1;
    int nci[4];
#pragma unroll
    for (int f = 0; f < 4; f++) nci[f] = ldg(COL(m.nc, f) + i);
    // vis is not an input of this kernel: a warp whose fast pass flagged an
    // operand recomputes and overwrites its sums
    for (int pass = HP_FAST(4) ? 1 : 0; pass >= 0; pass--) {
        double c[8];
        unsigned bad = 0;
        if (pass) visc_face<1>(m, s, P, i, q, nci, c, bad, s.prr);
        else visc_face<0>(m, s, P, i, q, nci, c, bad, s.prr);
        double acc[8];
#pragma unroll
        for (int k = 0; k < 8; k++) acc[k] = 0.0;
#pragma unroll
        for (int f = 0; f < 4; f++)
#pragma unroll
            for (int k = 0; k < 8; k++) acc[k] = acc[k] + qshfl(c[k], f);
        if (active) {
            COL(s.vis, q)[i] = acc[q];
            COL(s.vis, q + 4)[i] = acc[q + 4];
        }
        if (!__any_sync(0xffffffffu, bad)) break;
    }
}
__global__ void __launch_bounds__(128, HP_VISC4_MINB) k_visc4(DevMesh m, DevState<R> s, DevParams P) {
    k_visc4_body(m, s, P, blockIdx.x);
}

// Eight lanes per cell: each warp takes one phase of 8 cells (warps 2w and
// 2w+1 the gas and the liquid of the same cells), lane q of a cell face q.
// The per-cell sums over faces 1..4 are assembled with shuffles as in
// k_visc4, so vis is identical to k_visc4's.  Splitting the phases halves
// each lane's live state, which raises the resident warps.
// LIST = 1: the cells of m.wcells (the FP64 wall layers) instead of all
// cells.
template <int LIST>
__device__ __forceinline__ void k_visc8_body(DevMesh m, DevState<R> s, DevParams P, int bid) {
    const long long gt = (long long)bid * blockDim.x + threadIdx.x;
    const int q = (int)(gt & 3);
    const int ph = (int)((gt >> 5) & 1);
    const int ncell = LIST ? m.nwall : m.neles;
    const long long c = ((gt >> 6) << 3) + ((gt & 31) >> 2);
    const bool valid = c < ncell;
    const int k = valid ? (int)c : ncell - 1;
    const int i = LIST ? ldg(m.wcells + k) : k;
    const bool active = valid && ldg(m.iblank + i) == 1;
    int nci[4];
#pragma unroll
    for (int f = 0; f < 4; f++) nci[f] = ldg(COL(m.nc, f) + i);
    for (int pass = HP_FAST(4) ? 1 : 0; pass >= 0; pass--) {
        double c[4];
        unsigned bad = 0;
        if (pass) visc_face_ph<1>(m, s, P, i, q, nci, ph, c, bad, s.prr);
        else visc_face_ph<0>(m, s, P, i, q, nci, ph, c, bad, s.prr);
        double acc[4];
#pragma unroll
        for (int k = 0; k < 4; k++) acc[k] = 0.0;
#pragma unroll
        for (int f = 0; f < 4; f++)
#pragma unroll
            for (int k = 0; k < 4; k++) acc[k] = acc[k] + qshfl(c[k], f);
        if (active) COL(s.vis, 4 * ph + q)[i] = acc[q];
        if (!__any_sync(0xffffffffu, bad)) break;
    }
}
template <int LIST>
__global__ void __launch_bounds__(128, HP_VISC8_MINB) k_visc8(DevMesh m, DevState<R> s, DevParams P) {
    k_visc8_body<LIST>(m, s, P, blockIdx.x);
}

// Viscous fluxes once per face (FP32-arithmetic variants with a face list):
// the owner's contribution goes to the face record's first 8 values (the
// records are free until the first stage's k_faceflux); the other cell of an interior face takes its negative,
// since the face-centred stencil (both cells' neighbours), the face averages
// and the face vector are the same from either side up to the vector's sign.
__device__ __forceinline__ void k_facevisc_body(DevMesh m, DevState<R> s, DevParams P, int bid) {
    const int t = bid * blockDim.x + threadIdx.x;
    if (t >= m.nface) return;
    const int i = ldg(m.f_i + t), f = ldg(m.f_code + t) & 3;
    if (wall_face(m, i, f)) return;
    int nci[4];
#pragma unroll
    for (int k = 0; k < 4; k++) nci[k] = ldg(COL(m.nc, k) + i);
    double c[8];
    unsigned bad = 0;
    visc_face<0>(m, s, P, i, f, nci, c, bad, s.prr);
    R rec[FACE_REC];
#pragma unroll
    for (int k = 0; k < 8; k++) rec[k] = (R)c[k];
#pragma unroll
    for (int k = 8; k < FACE_REC; k++) rec[k] = R(0);
    store_frec(s.ff + (size_t)FACE_REC * (size_t)t, rec);
}
__global__ void __launch_bounds__(128, HP_VISC4_MINB) k_facevisc(DevMesh m, DevState<R> s, DevParams P) {
    k_facevisc_body(m, s, P, blockIdx.x);
}

// Per-cell viscous sums from k_facevisc's face values, in face order 1..4.
template <bool NC = true>
__device__ __forceinline__ void k_vis_gather_body(DevMesh m, DevState<R> s, int bid) {
    const int i = bid * blockDim.x + threadIdx.x;
    if (i >= m.neles) return;
    if (ldg(m.iblank + i) != 1) return;
    if (sizeof(R) != sizeof(double) && m.nwall > 0 && ldg(m.wclass + i)) return;   // FP64 wall layers
    double acc[8];
#pragma unroll
    for (int k = 0; k < 8; k++) acc[k] = 0.0;
#pragma unroll
    for (int f = 0; f < 4; f++) {
        const int code = ldg(COL(m.cface, f) + i);
        const size_t fid = (size_t)((code > 0 ? code : -code) - 1);
        const double sg = code > 0 ? 1.0 : -1.0;
        R rec[FACE_REC];
        load_frec<NC>(s.ff + (size_t)FACE_REC * fid, rec);
#pragma unroll
        for (int k = 0; k < 8; k++) acc[k] = acc[k] + sg * (double)rec[k];
    }
#pragma unroll
    for (int k = 0; k < 8; k++) COL(s.vis, k)[i] = acc[k];
}
__global__ void __launch_bounds__(256) k_vis_gather(DevMesh m, DevState<R> s) {
    k_vis_gather_body<true>(m, s, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Overset fringe cells take the barycentric combination of their four donor
// cells' conserved state after every RK stage (table from hp_overset_build).
// Donors are field cells, never fringe cells, so the updates are independent.
__global__ void __launch_bounds__(256) k_overset(DevMesh m, DevState<R> s) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m.nfringe) return;
    const int n = m.nfringe;
    const int i = ldg(m.fr + t);
    const int d0 = ldg(m.fdon + t), d1 = ldg(m.fdon + n + t), d2 = ldg(m.fdon + 2 * n + t),
              d3 = ldg(m.fdon + 3 * n + t);
    const double w0 = ldg(m.fw + t), w1 = ldg(m.fw + n + t), w2 = ldg(m.fw + 2 * n + t), w3 = ldg(m.fw + 3 * n + t);
    double v[10];
#pragma unroll
    for (int k = 0; k < 10; k++) {
        const double* c = COL(s.cn, k);
        v[k] = w0 * c[d0] + w1 * c[d1] + w2 * c[d2] + w3 * c[d3];
    }
#pragma unroll
    for (int k = 0; k < 10; k++) COL(s.cn, k)[i] = v[k];
}

// Partition halo: each halo cell takes the conserved state of the cell that
// owns it in another part of the batch, after every RK stage.  Destinations
// are halo cells, which no RK update writes; sources are owned cells.
__global__ void __launch_bounds__(256) k_halo(DevMesh m, DevState<R> s) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m.nhalo) return;
    const int i = ldg(m.hdst + t), j = ldg(m.hsrc + t);
#pragma unroll
    for (int k = 0; k < 10; k++) COL(s.cn, k)[i] = COL(s.cn, k)[j];
}

// ---------------------------------------------------------------------------
// Five-phase model: three dispersed, incompressible phases q, r, s (conserved
// columns 10-13, 14-17, 18-21: mass and momentum at densities rhod), carried
// by central fluxes with JST dissipation and coupled to the liquid by drag
// (src/sr_jamesonqrs.F90, src/sr_dissipationqrs.F90, src/sr_sourceqrs.F90).
// FP64 in every variant that accepts the model.

// JST switches (liquid pressure, liquid mass and each dispersed mass) and
// the Laplacian of columns 10-21, src/sr_dissipationqrs.F90:16-52; ghost
// neighbours read their parent through snb, as the reference copies them.
__global__ void __launch_bounds__(256) k_qrs_diss1(DevMesh m, DevState<R> s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.neles) return;
    const int a = ldg(COL(m.snb, 0) + i), b = ldg(COL(m.snb, 1) + i);
    const int c = ldg(COL(m.snb, 2) + i), d = ldg(COL(m.snb, 3) + i);
    const double e16 = (double)1.0e-16f;      // a REAL(4) literal in the reference
    const double* pp = COL(s.pr, P_PP);
    const double ppi = pp[i], ppa = pp[a], ppb = pp[b], ppc = pp[c], ppd = pp[d];
    double anun = fabs(ppa - ppi) + fabs(ppb - ppi) + fabs(ppc - ppi) + fabs(ppd - ppi);
    double anud = fabs(ppa + ppi) + fabs(ppb + ppi) + fabs(ppc + ppi) + fabs(ppd + ppi);
    double anupp = anun / anud;
    double sw[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
        const double* col = COL(s.cn, t == 0 ? 5 : 6 + 4 * t);    // cn(:,6), cn(:,11), cn(:,15), cn(:,19)
        const double v0 = col[i], v1 = col[a], v2 = col[b], v3 = col[c], v4 = col[d];
        anun = fabs(v1 - v0) + fabs(v2 - v0) + fabs(v3 - v0) + fabs(v4 - v0);
        anud = fabs(v1 + v0) + fabs(v2 + v0) + fabs(v3 + v0) + fabs(v4 + v0);
        sw[t] = anun / (anud + e16);
    }
    anupp = anupp + sw[0];
    double lap[12];
#pragma unroll
    for (int k = 0; k < 12; k++) {
        const double* col = COL(s.cn, 10 + k);
        const double v0 = col[i];
        lap[k] = col[a] - v0 + col[b] - v0 + col[c] - v0 + col[d] - v0;
    }
#pragma unroll
    for (int k = 0; k < 12; k++) COL(s.d2q, 10 + k)[i] = lap[k];
#pragma unroll
    for (int t = 0; t < 3; t++) COL(s.anuq, t)[i] = anupp + sw[1 + t];
}

// d24 of columns 10-21, src/sr_dissipationqrs.F90:62-157.
__global__ void __launch_bounds__(256) k_qrs_diss2(DevMesh m, DevState<R> s, DevParams P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.neles) return;
    const double dt = s.s[case_of(m, i)].dt;
    int nb[4];
#pragma unroll
    for (int f = 0; f < 4; f++) nb[f] = ldg(COL(m.snb, f) + i);
    const double vi = ldg(m.vol + i) / dt;
    double d24nc[4], out[12];
#pragma unroll
    for (int f = 0; f < 4; f++) d24nc[f] = 0.5 * (vi + ldg(m.vol + nb[f]) / dt);
#pragma unroll
    for (int set = 0; set < 3; set++) {
        const double* anu = COL(s.anuq, set);
        const double ai = anu[i];
        double d2c[4], d4c[4];
#pragma unroll
        for (int f = 0; f < 4; f++) {
            const double e2 = P.co2 * mx2(ai, anu[nb[f]]);
            const double e4 = mx2(0.0, P.co4 - e2);
            d2c[f] = e2 * d24nc[f];
            d4c[f] = e4 * d24nc[f];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const double* cn = COL(s.cn, 10 + 4 * set + k);
            const double* dq = COL(s.d2q, 10 + 4 * set + k);
            const double ci = cn[i], qi = dq[i];
            const double d2 = d2c[0] * (cn[nb[0]] - ci) + d2c[1] * (cn[nb[1]] - ci) + d2c[2] * (cn[nb[2]] - ci) +
                              d2c[3] * (cn[nb[3]] - ci);
            const double d4 = d4c[0] * (dq[nb[0]] - qi) + d4c[1] * (dq[nb[1]] - qi) + d4c[2] * (dq[nb[2]] - qi) +
                              d4c[3] * (dq[nb[3]] - qi);
            out[4 * set + k] = d2 - d4;
        }
    }
#pragma unroll
    for (int k = 0; k < 12; k++) COL(s.d24, 10 + k)[i] = out[k];
}

// src/sr_jamesonqrs.F90:21-60: dispersed fractions from their masses,
// renormalised with the two-phase fractions of this stage, velocities, and
// the masses and momenta rewritten from them; active elements.  (The
// reference also renormalises phig and phip there; nothing reads those
// values before the next primitive recovery overwrites them.)
__global__ void __launch_bounds__(256) k_qrs_prim(DevMesh m, DevState<R> s, DevParams P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.neles || ldg(m.iblank + i) != 1) return;
    const double emin = P.emin;
    double phd[3], u[3], v[3], w[3];
#pragma unroll
    for (int d = 0; d < 3; d++) phd[d] = mn2(mx2(COL(s.cn, 10 + 4 * d)[i] / P.rhod[d], emin), 1.0 - emin);
    const double phitotal = COL(s.pr, P_PHIG)[i] + COL(s.pr, P_PHIP)[i] + phd[0] + phd[1] + phd[2];
#pragma unroll
    for (int d = 0; d < 3; d++) phd[d] = phd[d] / phitotal;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double mass = COL(s.cn, 10 + 4 * d)[i];
        u[d] = COL(s.cn, 11 + 4 * d)[i] / mass;
        v[d] = COL(s.cn, 12 + 4 * d)[i] / mass;
        w[d] = COL(s.cn, 13 + 4 * d)[i] / mass;
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double r = P.rhod[d];
        COL(s.cn, 10 + 4 * d)[i] = phd[d] * r;
        COL(s.cn, 11 + 4 * d)[i] = phd[d] * r * u[d];
        COL(s.cn, 12 + 4 * d)[i] = phd[d] * r * v[d];
        COL(s.cn, 13 + 4 * d)[i] = phd[d] * r * w[d];
        COL(s.qpr, 4 * d)[i] = phd[d];
        COL(s.qpr, 4 * d + 1)[i] = u[d];
        COL(s.qpr, 4 * d + 2)[i] = v[d];
        COL(s.qpr, 4 * d + 3)[i] = w[d];
    }
}

// src/sr_jamesonqrs.F90:67-147: ghost states of the dispersed phases (inflow
// 2: fraction epslnmin at the liquid's ghost velocity; outflow 3: the
// parent's; wall 5: the parent's fraction, velocity reversed; other types
// keep their previous ghost state) and the ghost masses and momenta.  One
// thread per ghost (meshes without aliased ghost ids).
__global__ void __launch_bounds__(256) k_qrs_bc(DevMesh m, DevState<R> s, DevParams P) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= m.nghosts) return;
    const int np = m.g_par[g], ng = m.g_id[g], nt = m.g_type[g];
#pragma unroll
    for (int k = 10; k < 22; k++) COL(s.cn, k)[ng] = COL(s.cn, k)[np];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double* ph = COL(s.qpr, 4 * d);
        double* u = COL(s.qpr, 4 * d + 1);
        double* v = COL(s.qpr, 4 * d + 2);
        double* w = COL(s.qpr, 4 * d + 3);
        if (nt == 2) {
            ph[ng] = P.emin;
            u[ng] = COL(s.pr, P_UP)[ng]; v[ng] = COL(s.pr, P_VP)[ng]; w[ng] = COL(s.pr, P_WP)[ng];
        } else if (nt == 3) {
            ph[ng] = ph[np]; u[ng] = u[np]; v[ng] = v[np]; w[ng] = w[np];
        } else if (nt == 5) {
            ph[ng] = ph[np]; u[ng] = -u[np]; v[ng] = -v[np]; w[ng] = -w[np];
        }
        const double r = P.rhod[d];
        COL(s.cn, 10 + 4 * d)[ng] = ph[ng] * r;
        COL(s.cn, 11 + 4 * d)[ng] = ph[ng] * r * u[ng];
        COL(s.cn, 12 + 4 * d)[ng] = ph[ng] * r * v[ng];
        COL(s.cn, 13 + 4 * d)[ng] = ph[ng] * r * w[ng];
    }
}

// Central fluxes of the dispersed phases over the 4 faces in face order (none
// through type-5 walls), src/sr_jamesonqrs.F90:151-330; their drag with the
// liquid, src/sr_sourceqrs.F90:42-199 (constant liquid viscosity 0.001 of the
// AMUP_CONSTANT build), whose liquid-momentum terms go to qdrag for the flux
// kernel to add in the reference's order; then the RK stage update of
// columns 10-21 (src/sr_RK.F90).  Active elements.
__global__ void __launch_bounds__(128) k_qrs_flux(DevMesh m, DevState<R> s, DevParams P, int stage) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.neles || ldg(m.iblank + i) != 1) return;
    const unsigned kinds = ldg(m.fk + i);
    double rhs[12];
#pragma unroll
    for (int k = 0; k < 12; k++) rhs[k] = 0.0;
    double phi[3], ui[3], vi[3], wi[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        phi[d] = COL(s.qpr, 4 * d)[i]; ui[d] = COL(s.qpr, 4 * d + 1)[i];
        vi[d] = COL(s.qpr, 4 * d + 2)[i]; wi[d] = COL(s.qpr, 4 * d + 3)[i];
    }
#pragma unroll 1
    for (int f = 0; f < 4; f++) {
        if ((kinds >> (4 * f)) & FK_WALL) continue;
        const int n = ldg(COL(m.nc, f) + i);
        const double scx = ldg(COL(m.sc, 3 * f) + i), scy = ldg(COL(m.sc, 3 * f + 1) + i),
                     scz = ldg(COL(m.sc, 3 * f + 2) + i);
        const double area = sqrt(scx * scx + scy * scy + scz * scz);
        const double enx = scx / area, eny = scy / area, enz = scz / area;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double un = COL(s.qpr, 4 * d + 1)[n], vn = COL(s.qpr, 4 * d + 2)[n], wn = COL(s.qpr, 4 * d + 3)[n];
            const double qnl = ui[d] * enx + vi[d] * eny + wi[d] * enz;
            const double qnr = un * enx + vn * eny + wn * enz;
            const double phih = (phi[d] + COL(s.qpr, 4 * d)[n]) * 0.5;
            const double roh = (P.rhod[d] + P.rhod[d]) * 0.5;
            const double uh = (ui[d] + un) * 0.5, vh = (vi[d] + vn) * 0.5, wh = (wi[d] + wn) * 0.5;
            const double qh = (qnl + qnr) * 0.5;
            rhs[4 * d] = rhs[4 * d] + (phih * roh * qh) * area;
            rhs[4 * d + 1] = rhs[4 * d + 1] + (phih * roh * qh * uh) * area;
            rhs[4 * d + 2] = rhs[4 * d + 2] + (phih * roh * qh * vh) * area;
            rhs[4 * d + 3] = rhs[4 * d + 3] + (phih * roh * qh * wh) * area;
        }
    }
    // drag (Schiller-Naumann-type coefficient of the reference)
    const double voli = ldg(m.vol + i);
    const double up = COL(s.pr, P_UP)[i], vp = COL(s.pr, P_VP)[i], wp = COL(s.pr, P_WP)[i];
    const double amup = 0.001, gravity = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double du = up - ui[d], dv = vp - vi[d], dw = wp - wi[d];
        const double reyn = mx2(P.rhod[d] * 2.0 * P.radd[d] * sqrt(du * du + dv * dv + dw * dw) / amup, 0.001);
        const double relv = sqrt(du * du + dv * dv + dw * dw);
        double cd;
        if (reyn < 0.1) cd = 24.0 / reyn;
        else if (reyn < 1000.0) cd = 0.48 + 28.0 / pow(reyn, 0.85);
        else cd = 0.48;
        const double drag = 0.5 * cd * P.rhod[d] * 3.1415926 * P.radd[d] * P.radd[d] * relv * (phi[d] / P.vold[d]);
        rhs[4 * d + 1] = rhs[4 * d + 1] - drag * du * voli;
        rhs[4 * d + 2] = rhs[4 * d + 2] - drag * dv * voli - phi[d] * P.rhod[d] * gravity * voli;
        rhs[4 * d + 3] = rhs[4 * d + 3] - drag * dw * voli;
        COL(s.qdrag, 3 * d)[i] = drag * du * voli;
        COL(s.qdrag, 3 * d + 1)[i] = drag * dv * voli;
        COL(s.qdrag, 3 * d + 2)[i] = drag * dw * voli;
    }
    const double dtbyvol = s.s[case_of(m, i)].dt / voli;
#pragma unroll
    for (int k = 0; k < 12; k++) {
        const int j = 10 + k;
        const double r = rhs[k] - COL(s.d24, j)[i];
        const double cu = COL(s.cu, j)[i];
        double* cnp = COL(s.cn, j) + i;
        if (P.rk_scheme == 0) {
            if (stage == 1) {
                const double v = cu - (11.0 / 20.0) * dtbyvol * r;
                *cnp = v;
                COL(s.cn1, j)[i] = v;
            } else {
                const double upd = *cnp - (11.0 / 20.0) * dtbyvol * r;
                if (stage == 2) *cnp = (3.0 / 8.0) * cu + (5.0 / 8.0) * upd;
                else if (stage == 3) *cnp = (4.0 / 9.0) * cu + (5.0 / 9.0) * upd;
                else *cnp = (111.0 / 1331.0) * cu + (260.0 / 1331.0) * COL(s.cn1, j)[i] + (960.0 / 1331.0) * upd;
            }
        } else {
            if (stage == 1) *cnp = cu - dtbyvol * r;
            else {
                const double upd = *cnp - dtbyvol * r;
                if (stage == 2) *cnp = 0.75 * cu + 0.25 * upd;
                else *cnp = (1.0 / 3.0) * cu + (2.0 / 3.0) * upd;
            }
        }
    }
}

static inline unsigned grid_for(long long n, int block) {
    return (unsigned)((n + block - 1) / block);
}

#define MARK(k) do { if (hook && hook->mark) hook->mark(hook->ctx, (k)); } while (0)
#define EXCHANGE(p) do { if (hook && hook->exchange) hook->exchange(hook->xctx, (p)); } while (0)

// residual + RK update of one stage with Riemann solver Z (see face_eval)
template <int Z>
static void enqueue_flux(const DevMesh& m, const DevState<R>& s, const DevParams& P, cudaStream_t st, int stage,
                         const StepHook* hook) {
    const int b = 128;
    const unsigned gf = grid_for(m.neles, b), g4 = grid_for(4ll * m.neles, 128);
    if (m.aliased) {
        k_flux<true, false, Z><<<gf, b, 0, st>>>(m, s, P, stage);
        MARK(KK_SERIAL);
        k_flux_carry<Z><<<1, 1, 0, st>>>(m, s, P);
    } else if (sizeof(R) != sizeof(double) && m.nface > 0 && m.face_mode >= 2) {
        cudaMemsetAsync(s.racc, 0, 10 * (size_t)m.ld * sizeof(double), st);
        if (m.face_mode == 3) {
            k_facescatter<Z, true><<<grid_for(m.nface, 128), 128, 0, st>>>(m, s, P, m.fcolor, m.nface);
        } else {
            for (int c = 0; c < m.ncolor; c++) {
                const int n = m.fcoff[c + 1] - m.fcoff[c];
                k_facescatter<Z, false><<<grid_for(n, 128), 128, 0, st>>>(m, s, P, m.fcolor + m.fcoff[c], n);
            }
        }
        k_flux<false, false, Z, true><<<gf, 128, 0, st>>>(m, s, P, stage);
    } else if (sizeof(R) != sizeof(double) && m.nface > 0) {
        k_faceflux<Z><<<grid_for(m.nface, 128), 128, 0, st>>>(m, s, P);
        k_flux<false, true, Z><<<gf, 128, 0, st>>>(m, s, P, stage);
    } else {
        k_flux4<Z, 0><<<g4, 128, 0, st>>>(m, s, P, stage);
    }
}

static void enqueue_start(const DevMesh& m, const void* stp, const DevParams& P, cudaStream_t st,
                          int block, const StepHook* hook) {
    const DevState<R>& s = *static_cast<const DevState<R>*>(stp);
    MARK(KK_PRIM_START);
    const int cb = block > 0 ? block : 256;
    k_prim<PM_START><<<grid_for(m.neles, cb), cb, 0, st>>>(m, s, P);
    MARK(KK_COUNT);
}

// One time step of src/main.F90:520-654 (after enqueue_start).
static void enqueue_step(const DevMesh& m, const void* stp, const DevParams& P, cudaStream_t st,
                         int block, const StepHook* hook) {
    const DevState<R>& s = *static_cast<const DevState<R>*>(stp);
    // one-thread-per-cell kernels: `block` threads per block (64..512,
    // 0 = 256); four-lane kernels and the one-thread kernels of aliased
    // meshes: 128 (their launch bounds)
    const int cb = block > 0 ? block : 256, b = 128;
    const unsigned ge = grid_for(m.neles, cb), gf = grid_for(m.neles, b);
    const unsigned gg = grid_for(m.nghosts > 0 ? m.nghosts : 1, cb);
    EXCHANGE(HP_X_DT);
    MARK(KK_STEP_BEGIN);
    if (m.nhalo > 0) k_step_begin<<<1, 128, 0, st>>>(s, P, m.ncase, 1);
    else k_step_begin<<<grid_for(m.ncase, 128), 128, 0, st>>>(s, P, m.ncase, 0);
    // JST dissipation, src/sr_smooth.F90 (once per step)
    if (m.aliased) { MARK(KK_SERIAL); k_smooth_copy_serial<<<1, 1, 0, st>>>(m, s, 0); }
    MARK(KK_SMOOTH1);
    const unsigned gj = HP_JST_SETS ? grid_for(2ll * m.neles, cb) : ge;   // two threads per cell
    k_smooth1<<<gj, cb, 0, st>>>(m, s);
    if (m.aliased) { MARK(KK_SERIAL); k_smooth_copy_serial<<<1, 1, 0, st>>>(m, s, 1); }
    MARK(KK_SMOOTH2);
    k_smooth2<<<ge, cb, 0, st>>>(m, s, P);
    if (P.five_phase) {   // src/main.F90:570-572
        MARK(KK_QRS);
        k_qrs_diss1<<<grid_for(m.neles, 256), 256, 0, st>>>(m, s);
        k_qrs_diss2<<<grid_for(m.neles, 256), 256, 0, st>>>(m, s, P);
    }
    // viscous fluxes, src/sr_viscousgp.F90 (stage 1 of each step)
    if (m.nghosts > 0) {
        MARK(KK_BC_VISC);
        if (m.aliased) k_bc_serial<true><<<1, 1, 0, st>>>(m, s, P);
        else k_bc<true><<<gg, cb, 0, st>>>(m, s, P);
    }
    const unsigned g4 = grid_for(4ll * m.neles, 128);
    if (!P.inviscid) {
        MARK(KK_VISC);
        if (m.aliased) {
            k_visc<<<gf, b, 0, st>>>(m, s, P);
        } else if (sizeof(R) != sizeof(double) && HP_FACE_VISC && m.nface > 0) {
            k_facevisc<<<grid_for(m.nface, 128), 128, 0, st>>>(m, s, P);
            k_vis_gather<<<grid_for(m.neles, 256), 256, 0, st>>>(m, s);
        } else if (HP_VISC_SPLIT) {
            k_visc8<0><<<grid_for(8ll * m.neles, 128), 128, 0, st>>>(m, s, P);
        } else {
            k_visc4<<<g4, 128, 0, st>>>(m, s, P);
        }
        // FP64 wall layers: their viscous sums replaced by FP64 ones
        if (sizeof(R) != sizeof(double) && m.nwall > 0) wall_fp64.visc(m, fp64_view(s), P, st);
    }
    for (int stage = 1; stage <= P.nstage; stage++) {
        // src/sr_hllcbatten.F90:29-33: primitiveplusbc, derivative, limiter
        MARK(KK_PRIM_STAGE);
        k_prim<PM_STAGE><<<ge, cb, 0, st>>>(m, s, P);
        if (m.nghosts > 0) {
            MARK(KK_BC);
            if (m.aliased) k_bc_serial<false><<<1, 1, 0, st>>>(m, s, P);
            else k_bc<false><<<gg, cb, 0, st>>>(m, s, P);
        }
        // (the Jameson flux reads no gradients: src/sr_jameson.F90:24 calls
        // primitiveplusbc only)
        if (P.myorder == 2 && P.myflux != 3) {
            MARK(KK_GRAD);
            if (m.aliased) k_grad<false><<<gf, b, 0, st>>>(m, s, P);
            else if (sizeof(R) != sizeof(double)) k_grad<true><<<gf, b, 0, st>>>(m, s, P);
            else k_grad4<0><<<g4, 128, 0, st>>>(m, s, P);
            if (m.aliased) { MARK(KK_SERIAL); k_phi_copy_serial<<<1, 1, 0, st>>>(m, s); }
            // FP64 wall layers: FP64 gradients and limiter of those cells and
            // their neighbours, for the FP64 fluxes below
            if (sizeof(R) != sizeof(double) && m.nwall > 0) wall_fp64.grad(m, fp64_view(s), P, st);
        }
        if (P.five_phase) {   // src/mod_Fluxmodule.F90:18-20: jamesonqrs (and sourceqrs)
            MARK(KK_QRS);
            k_qrs_prim<<<grid_for(m.neles, 256), 256, 0, st>>>(m, s, P);
            if (m.nghosts > 0) k_qrs_bc<<<grid_for(m.nghosts, 256), 256, 0, st>>>(m, s, P);
            k_qrs_flux<<<grid_for(m.neles, 128), 128, 0, st>>>(m, s, P, stage);
        }
        MARK(KK_FLUX);
        if (P.myflux == 1) enqueue_flux<1>(m, s, P, st, stage, hook);
        else if (P.myflux == 3) enqueue_flux<2>(m, s, P, st, stage, hook);
        else enqueue_flux<0>(m, s, P, st, stage, hook);
        // FP64 wall layers: their fluxes, sources and RK update (the FP32
        // kernels above left those cells alone)
        if (sizeof(R) != sizeof(double) && m.nwall > 0) wall_fp64.flux(m, fp64_view(s), P, st, stage);
        if (m.nfringe > 0) {
            MARK(KK_OVERSET);
            k_overset<<<grid_for(m.nfringe, 256), 256, 0, st>>>(m, s);
        }
        if (m.nhalo > 0) {
            MARK(KK_HALO);
            k_halo<<<grid_for(m.nhalo, 256), 256, 0, st>>>(m, s);
        }
        EXCHANGE(HP_X_HALO);
    }
    // src/main.F90:595-641: primitive, residual norms, cu = cn
    MARK(KK_PRIM_END);
    k_prim<PM_END><<<ge, cb, 0, st>>>(m, s, P);
    MARK(KK_STEP_END);
    k_step_end<<<grid_for(m.ncase, 128), 128, 0, st>>>(s, m.ncase);
    // start of the next step: primitive + dt contributions
    MARK(KK_PRIM_START);
    k_prim<PM_START><<<ge, cb, 0, st>>>(m, s, P);
    MARK(KK_COUNT);
}
#undef MARK
#undef EXCHANGE

// ---------------------------------------------------------------------------
// Fused step: one cooperative launch runs a whole time step.  The kernels of
// enqueue_step run as phases, in the same order and with the same bodies,
// over virtual blocks of 128 threads; a grid-wide barrier separates the
// phases.  Results are those of the separate launches bit for bit (every
// reduction is order-free: min, max, integer sums).  For small meshes, where
// the fixed cost of ~20 dependent launches is a large part of a step.
// Not for aliased meshes, the five-phase model, face modes 2 and 3, overset
// fringes, partition halos or FP64 wall layers (the host keeps the graph).
// Built in the parity variant only (HP_FUSED_STEP): without FMA contraction
// the bodies round the same inlined here as in their own kernels.

#if HP_FUSED_STEP
#ifndef HP_FUSED_MINB
#define HP_FUSED_MINB 4
#endif
// spins of a barrier wait (each with a 64 ns sleep) before it gives up
#ifndef HP_SYNC_SPIN_LIMIT
#define HP_SYNC_SPIN_LIMIT (1ll << 24)
#endif

// Every block of the grid arrives; false once any wait of any block gave up
// (then every block returns at its next barrier, whose waits are bounded).
__device__ __forceinline__ bool grid_sync(GridSync* g) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &g->gen;
        const unsigned gen0 = *vgen;
        __threadfence();
        int ok = 1;
        if (atomicAdd(&g->count, 1u) == gridDim.x - 1) {
            atomicExch(&g->count, 0u);
            __threadfence();
            atomicAdd(&g->gen, 1u);
        } else {
            long long it = 0;
            while (*vgen == gen0) {
                if (++it > HP_SYNC_SPIN_LIMIT) {
                    atomicExch(&g->err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok_s = ok && *(volatile int*)&g->err == 0;
    }
    __syncthreads();
    return ok_s != 0;
}

template <int Z>
__global__ void __launch_bounds__(128, HP_FUSED_MINB) k_step_fused(DevMesh m, DevState<R> s, DevParams P,
                                                                   GridSync* g) {
    const int nb = gridDim.x;
#define PHASE(nthreads, CALL) \
    for (int vb = blockIdx.x; vb < (int)(((long long)(nthreads) + 127) / 128); vb += nb) { CALL; }
#define SYNC \
    if (!grid_sync(g)) return;
    // src/main.F90:521-556: dt and time of every case
    PHASE(m.ncase, { const int c = vb * 128 + threadIdx.x; if (c < m.ncase) step_begin_case(s.s + c, P, s.s[c].dtmin_bits); })
    SYNC
    PHASE(m.neles, k_smooth1_body(m, s, vb))
    SYNC
    PHASE(m.neles, k_smooth2_body(m, s, P, vb))
    SYNC
    if (m.nghosts > 0) {
        PHASE(m.nghosts, k_bc_body<true>(m, s, P, vb))
        SYNC
    }
    if (!P.inviscid) {
        if (sizeof(R) != sizeof(double) && HP_FACE_VISC && m.nface > 0) {
            PHASE(m.nface, k_facevisc_body(m, s, P, vb))
            SYNC
            PHASE(m.neles, k_vis_gather_body<false>(m, s, vb))
        } else if (HP_VISC_SPLIT) {
            PHASE(8ll * m.neles, k_visc8_body<0>(m, s, P, vb))
        } else {
            PHASE(4ll * m.neles, k_visc4_body(m, s, P, vb))
        }
        SYNC
    }
    for (int stage = 1; stage <= P.nstage; stage++) {
        // the primitive pass reduces through shared memory: a block barrier
        // between its virtual blocks
        PHASE(m.neles, { k_prim_body<PM_STAGE>(m, s, P, vb); __syncthreads(); })
        SYNC
        if (m.nghosts > 0) {
            PHASE(m.nghosts, k_bc_body<false>(m, s, P, vb))
            SYNC
        }
        if (P.myorder == 2) {
            if (sizeof(R) != sizeof(double)) {
                PHASE(m.neles, k_grad_body<true>(m, s, P, vb))
            } else {
                PHASE(4ll * m.neles, k_grad4_body<0>(m, s, P, vb))
            }
            SYNC
        }
        if (sizeof(R) != sizeof(double) && m.nface > 0) {
            PHASE(m.nface, (k_faceflux_body<Z, false>(m, s, P, vb)))
            SYNC
            PHASE(m.neles, (k_flux_body<false, true, Z, false, false>(m, s, P, stage, vb)))
        } else {
            PHASE(4ll * m.neles, (k_flux4_body<Z, 0, false>(m, s, P, stage, vb)))
        }
        SYNC
    }
    PHASE(m.neles, { k_prim_body<PM_END>(m, s, P, vb); __syncthreads(); })
    SYNC
    PHASE(m.ncase, k_step_end_body(s, m.ncase, vb))
    SYNC
    PHASE(m.neles, { k_prim_body<PM_START>(m, s, P, vb); __syncthreads(); })
#undef PHASE
#undef SYNC
}

// Blocks of the fused step on this device: as many as are co-resident
// (cooperative launch), at most the largest phase's virtual blocks.
static int fused_grid(const DevMesh& m, const DevParams& P) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 0;
    cudaError_t e = P.myflux == 1
                        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_fused<1>, 128, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_fused<0>, 128, 0);
    if (e != cudaSuccess || per_sm < 1) return 0;
    const long long need = (8ll * m.neles + 127) / 128;
    return (int)std::min<long long>((long long)sms * per_sm, std::max(need, 1ll));
}

static cudaError_t enqueue_fused(const DevMesh& m, const void* stp, const DevParams& P, cudaStream_t st,
                                 GridSync* sync, int grid) {
    DevState<R> s = *static_cast<const DevState<R>*>(stp);
    DevMesh mm = m;
    DevParams pp = P;
    void* args[] = {&mm, &s, &pp, &sync};
    return P.myflux == 1 ? cudaLaunchCooperativeKernel((void*)k_step_fused<1>, grid, 128, args, 0, st)
                         : cudaLaunchCooperativeKernel((void*)k_step_fused<0>, grid, 128, args, 0, st);
}
#else
// variants without the fused step (built with FMA contraction)
static int fused_grid(const DevMesh&, const DevParams&) { return 0; }
static cudaError_t enqueue_fused(const DevMesh&, const void*, const DevParams&, cudaStream_t, GridSync*, int) {
    return cudaErrorNotSupported;
}
#endif

}  // namespace HP_NS
}  // namespace hp
