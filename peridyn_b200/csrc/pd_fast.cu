// pd_fast.cu -- throughput modes PD_PREC_FP32C and PD_PREC_FP64.
//
// One launch per velocity-Verlet step (two for state-based blocks): the
// thread of particle p gathers p's bond forces once (no serial replay), and
// then, still in registers, applies the second half kick, the boundary
// velocities, the next step's half kick, the drift and the boundary
// positions, writing the next displacement into the other half of a double
// buffer that neighbours read in the next launch.
//
// FP32C: bond arithmetic in FP32 on FP32 displacements u = y - x, with the
// cancellation-free extension e = (2 xi.eta + eta.eta) / (|xi+eta| + |xi|);
// positions are accumulated in FP64 (u64) and rounded to FP32 once per step.
// Reference positions are stored in FP32 relative to the block's centre.
// FP64: the same single-pass algorithm in FP64 throughout.
//
// Per bond (general_material.jl:332-362 restated with the identities
// w|xi| = 1 and e*w = s):
//   s   = e / |xi|                          (break when s >= cs)
//   PMB t = c s                             (bond_based.jl:195-231)
//   LPS t = (3K-5G)(theta_p/m_p + theta_q/m_q) + 15G s (1/m_p + 1/m_q)
//                                           (ordinary_state_based.jl:176-187)
//   f_p += (t / (2|Y|)) V_q Y  ... scaled by 1/rho_p once per particle.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "pd_env_impl.h"

namespace pd {
namespace {

constexpr int kT = 128;
inline unsigned gridn(int64_t n, int t = kT) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

template <class R>
struct Tr;
template <>
struct Tr<float> {
    using V4 = float4;
    using V2 = float2;
    static __device__ __forceinline__ float rsq(float a) { return rsqrtf(a); }
    static __device__ __forceinline__ float fma_(float a, float b, float c) { return fmaf(a, b, c); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
    // single-instruction approximations (relative error of order 2^-22)
    static __device__ __forceinline__ float sqrt_(float a) {
        float r;
        asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
        return r;
    }
    static __device__ __forceinline__ float rcp(float a) {
        float r;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
        return r;
    }
    // One 256-bit load of a particle record (x, volume | u, -); the record
    // buffer is not written while a kernel reads it.
    // NC = false: a coherent load, for the persistent kernel, which reads
    // records other blocks wrote earlier in the same launch
    template <bool NC = true>
    static __device__ __forceinline__ void load_rec(const float4 *r, float4 &x, float4 &u) {
        if (NC)
            asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                : "=f"(x.x), "=f"(x.y), "=f"(x.z), "=f"(x.w), "=f"(u.x), "=f"(u.y), "=f"(u.z), "=f"(u.w)
                : "l"(r));
        else
            asm volatile("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=f"(x.x), "=f"(x.y), "=f"(x.z), "=f"(x.w), "=f"(u.x), "=f"(u.y), "=f"(u.z), "=f"(u.w)
                         : "l"(r));
    }
};
template <>
struct Tr<double> {
    using V4 = double4;
    using V2 = double2;
    static __device__ __forceinline__ double rsq(double a) { return rsqrt(a); }
    static __device__ __forceinline__ double fma_(double a, double b, double c) { return fma(a, b, c); }
    static __device__ __forceinline__ double div(double a, double b) { return a / b; }
    static __device__ __forceinline__ double sqrt_(double a) { return sqrt(a); }
    static __device__ __forceinline__ double rcp(double a) { return 1.0 / a; }
    template <bool NC = true>
    static __device__ __forceinline__ void load_rec(const double4 *r, double4 &x, double4 &u) {
        if (NC) {
            asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(x.x), "=d"(x.y), "=d"(x.z), "=d"(x.w) : "l"(r));
            asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(u.x), "=d"(u.y), "=d"(u.z), "=d"(u.w) : "l"(r + 1));
        } else {
            asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(x.x), "=d"(x.y), "=d"(x.z), "=d"(x.w)
                         : "l"(r));
            asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(u.x), "=d"(u.y), "=d"(u.z), "=d"(u.w)
                         : "l"(r + 1));
        }
    }
};

template <class R>
struct FBlock {
    int32_t kind, nt, pair_base, pad;
    R c11;
};
template <class R>
struct FPair {
    R cs, k35, g15;
    R psi;  // elasto-plastic: sqrt(2 psi), so that C = psi / sqrt(td_norm2)
};

constexpr int kMaxFastBC = 8;
struct FBC {
    int32_t kind, dims;
    double rate[3];
    double scale[3], fix[3];  // DeltaScale / ScaleFixWait
    double lo[3], hi[3];      // Container limits
    int32_t has_limits, pad;
    int64_t n;
    const int32_t *idx;  // ascending internal indices
    double4 *last;
    int64_t sn;          // ScaleFixWait scalebool particles
    const int32_t *sidx;
    int64_t rank_lo;     // rank[p - rank_lo]: position of particle p in idx / last
    const int32_t *rank;
};

template <class R>
struct StepArgs {
    int64_t N;
    // Interleaved particle records, double-buffered by step parity:
    // xu[2i] = (x, w) (FP32C: relative to the block centre; identical in
    // both buffers), xu[2i+1] = (u, w) displacement; w = the volume (times
    // c in bond-based blocks) in both halves.  One address per neighbour
    // fetches both.
    const typename Tr<R>::V4 *xu;
    typename Tr<R>::V4 *xn;  // next-step buffer (only the u records are written)
    double *ax, *ay, *az;    // FP64 displacement accumulator (FP32C)
    typename Tr<R>::V4 *v, *f, *p;
    const R *irho, *mass;
    typename Tr<R>::V2 *mab;  // (theta/m, 1/m) of state-based particles
    const int32_t *tinfo, *cnt, *nbr;
    const SliceInfo *si;
    // record staging plans (FP32C staged kernels): see pd_env
    const int32_t *splan_off, *splan, *spos;
    int32_t *serr;        // set when a staging copy did not land in time
    // elasto-plastic blocks: plastic strain per bond slot (read edp_in,
    // written edp_out), 1/sqrt(td_norm2) per particle, and per slot the
    // slot of the reverse bond in the neighbour's family
    const double *edp_in;
    double *edp_out;
    R *rtd;
    const int32_t *partner;
    int32_t ep;  // the environment has elasto-plastic blocks
    // contact accelerations of this step, added by the fused integration
    // (MODE 1/2; null without contacts)
    const typename Tr<R>::V4 *cacc;
    int32_t stage_bytes;  // dynamic shared memory of the staged kernels
    // Slice order of the one-slice-per-block kernels: with swz_g = G > 0,
    // block b = r + G c walks slice r K + c (K = swz_k), so blocks that are
    // dispatched G apart -- the ones sharing an SM -- walk consecutive
    // slices and share their neighbour records in L1.  0: block b walks
    // slice b.
    int32_t swz_g, swz_k;
    uint32_t *words;
    const FBlock<R> *fb;
    const FPair<R> *fp;
    const int32_t *deformed;
    int32_t all_def;  // every non-skip block has deformed (known on the host): deformed[] is not read
    const double4 *x64;
    const uint8_t *bcbits;
    R c;
    double dt;
    int64_t ts;  // time_step of the position BCs applied by this launch
    int nbc;
    uint32_t dir_vel, dir_pos;  // bit k set: BC k moves in the negative direction
    FBC bc[kMaxFastBC];
};


__device__ __forceinline__ double &cmp(double4 &a, int d) { return d == 0 ? a.x : (d == 1 ? a.y : a.z); }

// Work split of a 32-particle slice over WPS warps: warp w handles the
// contiguous slot range [w*per, (w+1)*per) of every particle of the slice,
// per = ceil(len / WPS) with len the slice's slot count, so a family of 92
// slots splits 23/23/23/23 over four warps.  Partial sums are combined in a
// fixed order, so results do not depend on scheduling.
template <int WPS>
struct Split {
    static constexpr int BT = WPS <= 4 ? 128 : 256;  // threads per block
    static constexpr int NW = BT / 32;                // warps per block
    static constexpr int SPB = NW / WPS;              // slices per block
    static constexpr int MINB = 1024 / BT;            // resident blocks per SM aimed for (<= 64 registers)
    // Two slots in flight fit 56 registers: 9 blocks of 128 threads per SM,
    // so 4 warps per slice cover 1332 slices in one wave instead of 1184.
    static constexpr int MINB_U2 = 1152 / BT;
    static constexpr int MINB_THETA = 1280 / BT;      // the dilatation walk fits 48 registers
};

// The index loads of a bond walk depend on nothing, but each thread only
// has a few of them in flight.  At kernel entry every warp of an
// explicit-index slice asks L2 for all 128-byte index lines of the chunks it
// will walk (one line per lane), so the walk's loads hit L2 instead of
// waiting on HBM one chunk at a time.  Stencil slices read no indices.
template <int WPS>
__device__ __forceinline__ void warp_range(int32_t len, int w, int32_t &k0, int32_t &k1) {
    const int32_t per = WPS == 1 ? len : (len + WPS - 1) / WPS;
    k0 = min(w * per, len);
    k1 = min(k0 + per, len);
}

template <int WPS>
__device__ __forceinline__ void prefetch_slice_indices(const int32_t *nbr, const SliceInfo *si, int64_t s, int w,
                                                       int lane) {
    const SliceInfo d = si[s];
    if (d.mode != kExplicit) return;
    int32_t k0, k1;
    warp_range<WPS>(d.len, w, k0, k1);
    for (int32_t k = k0 + lane; k < k1; k += 32) asm volatile("prefetch.global.L2 [%0];" ::"l"(nbr + d.nbr + 32 * (int64_t)k));
}

// Bits of the slots [w0, w0 + kend) of one intact word (kend <= 32 - (w0 & 31)),
// bit j <-> slot w0 + j.
__device__ __forceinline__ uint32_t range_bits(uint32_t word, int32_t w0, int32_t kend) {
    const uint32_t b = word >> (w0 & 31);
    return kend >= 32 ? b : (b & ((1u << kend) - 1u));
}

template <int SPB, class A>
__device__ __forceinline__ int64_t slice_of_block(const A &a) {
    const int64_t b = blockIdx.x;
    if (SPB != 1 || a.swz_g == 0) return b;
    return (b % a.swz_g) * a.swz_k + b / a.swz_g;
}

// Neighbour of slot j of a chunk: explicit slices store one index per
// (slot, lane); stencil slices one offset per slot, shared by the warp, so
// the 32 lanes gather 32 consecutive records.
template <bool ST>
__device__ __forceinline__ int32_t slot_neighbour(const int32_t *np, int32_t j, int64_t p) {
    return ST ? (int32_t)p + __ldg(np + j) : __ldg(np + 32 * j);
}

// Combine the WPS partial sums of one slice without a block barrier: each
// warp publishes its partials, and the last warp of the slice to arrive
// adds them in warp order (fixed, so the result does not depend on which
// warp arrives last) and continues with the particle update.  Returns
// true in the lanes of that warp.
template <int WPS, int NC, class R>
__device__ __forceinline__ bool last_arrival_sum(R (*sh)[NC][32], int *arrive, int wid, int lane, R *v) {
    const int w = wid % WPS, sl = wid / WPS;
#pragma unroll
    for (int c = 0; c < NC; ++c) sh[wid][c][lane] = v[c];
    __syncwarp();
    int old = 0;
    if (lane == 0) {
        __threadfence_block();
        old = atomicAdd(&arrive[sl], 1);
    }
    old = __shfl_sync(0xffffffffu, old, 0);
    if (old != WPS - 1) return false;
    __threadfence_block();
    if (lane == 0) arrive[sl] = 0;  // every warp of the slice has arrived: ready for reuse
    const int w0 = wid - w;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        R s = 0;
        for (int k = 0; k < WPS; ++k) s += sh[w0 + k][c][lane];
        v[c] = s;
    }
    return true;
}

// Gather of p's bonds in the chunks owned by warp w.  Returns the
// acceleration before the 1/rho scaling.  Every bond appears in both
// endpoint families and the serial loop adds its term to f_p from both
// visits, hence the factor 2 (t/|Y| rather than t/(2|Y|)).
// Bond kinematics from the neighbour record (xq, uq) and the negated own
// record (nx, nu): deformed bond vector Y = xi + eta, |xi|^2 and the
// cancellation-free stretch numerator num = eta . (xi + Y) = |Y|^2 - |xi|^2.
template <class R>
struct Kin {
    R Y0, Y1, Y2, xx2, num;
    // f += c Y
    __device__ __forceinline__ void accumulate(R c, R &fx, R &fy, R &fz) const {
        fx = Tr<R>::fma_(c, Y0, fx);
        fy = Tr<R>::fma_(c, Y1, fy);
        fz = Tr<R>::fma_(c, Y2, fz);
    }
    __device__ __forceinline__ Kin(const typename Tr<R>::V4 &xq, const typename Tr<R>::V4 &uq,
                                   const typename Tr<R>::V4 &nx, const typename Tr<R>::V4 &nu) {
        const R x0 = xq.x + nx.x, x1 = xq.y + nx.y, x2 = xq.z + nx.z;
        const R e0 = uq.x + nu.x, e1 = uq.y + nu.y, e2 = uq.z + nu.z;
        Y0 = x0 + e0;
        Y1 = x1 + e1;
        Y2 = x2 + e2;
        xx2 = Tr<R>::fma_(x2, x2, Tr<R>::fma_(x1, x1, x0 * x0));
        num = Tr<R>::fma_(e2, x2 + Y2, Tr<R>::fma_(e1, x1 + Y1, e0 * (x0 + Y0)));
    }
};
// FP32: the (x, y) components as packed f32x2 operations.
template <>
struct Kin<float> {
    float2 Yxy;
    float Y2, xx2, num;
    __device__ __forceinline__ void accumulate(float c, float2 &fxy, float &fz) const {
        fxy = __ffma2_rn(make_float2(c, c), Yxy, fxy);
        fz = fmaf(c, Y2, fz);
    }
    __device__ __forceinline__ Kin(const float4 &xq, const float4 &uq, const float4 &nx, const float4 &nu) {
        const float2 d = __fadd2_rn(make_float2(xq.x, xq.y), make_float2(nx.x, nx.y));
        const float2 e = __fadd2_rn(make_float2(uq.x, uq.y), make_float2(nu.x, nu.y));
        const float dz = xq.z + nx.z, ez = uq.z + nu.z;
        const float2 Y = __fadd2_rn(d, e);
        const float Yz = dz + ez;
        const float2 S = __fadd2_rn(d, Y);
        const float2 dd = __fmul2_rn(d, d);
        const float2 es = __fmul2_rn(e, S);
        xx2 = fmaf(dz, dz, dd.x + dd.y);
        num = fmaf(ez, dz + Yz, es.x + es.y);
        Yxy = Y;
        Y2 = Yz;
    }
};

// STG: the neighbour records come from the block's staged copy in shared
// memory (stg, lane 0's record of slot k at sp[k]) instead of global memory.
template <class R, int KIND, bool kBreak, int WPS, int U, bool ST, bool MULTI, bool NC = true, bool STG = false>
__device__ __forceinline__ void bond_walk(const StepArgs<R> &a, int64_t p, int32_t k0, int32_t k1, const int32_t *nb,
                                          uint32_t *wp, const FBlock<R> &B, int tp, const FPair<R> &pp0,
                                          typename Tr<R>::V4 xp, typename Tr<R>::V4 up, R Ap, R Bp, R &fx, R &fy,
                                          R &fz, const typename Tr<R>::V4 *stg = nullptr,
                                          const int32_t *sp = nullptr, R rtdp = R(0)) {
    using V4 = typename Tr<R>::V4;
    FPair<R> pp = pp0;  // the pair (type p, type p); MULTI reloads it per slot
    const V4 nx{-xp.x, -xp.y, -xp.z, R(0)}, nu{-up.x, -up.y, -up.z, R(0)};
    float2 fxy = make_float2(0.f, 0.f);  // FP32: packed (fx, fy)
    for (int32_t w0 = k0, wend; w0 < k1; w0 = wend) {
        // the part of [k0, k1) in one intact word
        wend = min(k1, (w0 | 31) + 1);
        uint32_t *wptr = wp + 32 * (w0 >> 5);
        const int32_t kend = wend - w0;
        const uint32_t bits = range_bits(*wptr, w0, kend);
        if (!bits) {
            if (KIND == PD_MAT_ELASTO_PLASTIC) {  // carry the strain of broken bonds
                const int64_t e0 = ((int64_t)(wptr - a.words) << 5) + (w0 & 31);
                for (int32_t j = 0; j < kend; ++j) a.edp_out[e0 + j] = a.edp_in[e0 + j];
            }
            continue;
        }
        // Dense, branch-free walk over the chunk: intact bonds dominate, so
        // every slot is evaluated and its term selected by its bit; the
        // unrolled iterations' index and neighbour loads overlap.  Empty
        // stencil slots point at an in-range record and carry a 0 bit.
        const int32_t *np = nb + (ST ? 1 : 32) * w0;
        const int32_t *spp = STG ? sp + w0 : nullptr;
        // elasto-plastic: per-slot state index of the chunk's first slot
        const int64_t ebase = KIND == PD_MAT_ELASTO_PLASTIC ? ((int64_t)(wptr - a.words) << 5) + (w0 & 31) : 0;
        uint32_t okm = 0, bit = 1u;  // okm: slots within the critical stretch
#pragma unroll U
        for (int32_t j = 0; j < kend; ++j, bit <<= 1) {
            const int32_t q = slot_neighbour<ST>(np, j, p);
            V4 xq, uq;
            if constexpr (STG) {
                const int32_t r = __ldg(spp + j) + (int32_t)(p & 31);
                xq = stg[2 * r];
                uq = stg[2 * r + 1];
            } else {
                Tr<R>::template load_rec<NC>(a.xu + 2 * (int64_t)q, xq, uq);
            }
            const Kin<R> k(xq, uq, nx, nu);
            const R num = k.num, xx2 = k.xx2;
            const R wq = xq.w;  // V_q (c V_q in bond-based blocks)
            // stretch s = num / dl;  |Y|^2 = |xi|^2 + num
            const R lx = Tr<R>::sqrt_(xx2), ly = Tr<R>::sqrt_(xx2 + num);
            const R dl = Tr<R>::fma_(ly, lx, xx2);  // (|Y| + |xi|) |xi|
            const bool live = (bits & bit) != 0u;
            if (MULTI && live) pp = a.fp[B.pair_base + tp + (a.tinfo[q] & 255) * B.nt];
            const bool ok = num < pp.cs * dl;
            if (kBreak) okm |= ok ? bit : 0u;
            // coef = t V / |Y| with t * dl accumulated in tn; bond-based
            // records carry c V in w (k_import), so tn = num there
            R tn;
            if (KIND == PD_MAT_BOND_BASED) {
                tn = num;
            } else if (KIND == PD_MAT_ORDINARY_STATE_BASED) {
                typename Tr<R>::V2 mq = a.mab[q];
                tn = Tr<R>::fma_(pp.k35 * (Ap + mq.x), dl, pp.g15 * num * (Bp + mq.y));
            } else {
                // force_density_t_ij (elasto_plastic.jl:215-242) of both
                // visits: p's (its slot e, its td_norm2) and q's (the
                // reverse slot, q's td_norm2); f_p gets (t_pq + t_qp) / 2.
                // With A = theta/m, B = 1/m: theta_ij = (A_p + A_q) /
                // (B_p + B_q), tn = 3K (A_p + A_q), td_trial = 15G w
                // (B_p + B_q) (ed - edp).
                typename Tr<R>::V2 mq = a.mab[q];
                const R As = Ap + mq.x, Bs = Bp + mq.y;
                const R ext = num * Tr<R>::rcp(ly + lx);
                const R ed = Tr<R>::fma_(-As * Tr<R>::rcp(Bs), lx * R(1.0 / 3.0), ext);
                const R gB = pp.g15 * Tr<R>::rcp(lx) * Bs;
                const int64_t e = ebase + j;
                const int32_t pe = a.partner[e];
                const double eo = a.edp_in[e];
                const R ede_p = ed - (R)eo, ede_q = ed - (R)a.edp_in[pe];
                const R Cp = pp.psi * rtdp, Cq = pp.psi * a.rtd[q];
                const bool pl = Cp <= R(1);  // p's visit yields
                const R td_p = gB * ede_p * (pl ? Cp : R(1));
                const R td_q = gB * ede_q * (Cq <= R(1) ? Cq : R(1));
                tn = Tr<R>::fma_(pp.k35, As, R(0.5) * (td_p + td_q)) * dl;
                a.edp_out[e] = (live && ok && pl) ? (double)Tr<R>::fma_(ede_p, R(1) - Cp, (R)eo) : eo;
            }
            const R coef = (live && ok) ? tn * wq * Tr<R>::rcp(dl * ly) : R(0);
            if constexpr (sizeof(R) == 4) k.accumulate(coef, fxy, fz);
            else k.accumulate(coef, fx, fy, fz);
        }
        // bonds break rarely; two warps may own parts of one word
        const uint32_t brk = bits & ~okm;
        if (kBreak && brk) atomicAnd(wptr, ~(brk << (w0 & 31)));
    }
    if constexpr (sizeof(R) == 4) {
        fx += fxy.x;
        fy += fxy.y;
    }
}

// U consecutive stencil offsets in one load.  p is 4 U-byte aligned: a
// slice's offsets start at a multiple of 32 entries, a warp's slot range at
// a multiple of 4 (len is a multiple of 32, split over 1, 2, 4 or 8 warps),
// and the walks step through it U slots at a time.
template <int U>
__device__ __forceinline__ void load_offsets(const int32_t *p, int32_t (&o)[U]) {
    if constexpr (U == 4) {
        const int4 v = __ldg(reinterpret_cast<const int4 *>(p));
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
        o[3] = v.w;
    } else if constexpr (U == 2) {
        const int2 v = __ldg(reinterpret_cast<const int2 *>(p));
        o[0] = v.x;
        o[1] = v.y;
    } else {
#pragma unroll
        for (int u = 0; u < U; ++u) o[u] = __ldg(p + u);
    }
}

// The stencil walk of bond_walk (bond-based and state-based blocks, records
// from global memory) with the slot offsets loaded one group of U slots
// ahead: the offsets of the next group are in flight while the current
// group's records are fetched, so a slot waits for one memory access (its
// record) instead of two in a row (offset, then record).  The neighbour of
// slot j is p + o_j (o_j shared by the warp), its record xb + 2 o_j.  Same
// arithmetic in the same slot order as bond_walk.
template <class R, int KIND, bool kBreak, int U, bool MULTI, bool NC>
__device__ __forceinline__ void bond_walk_st(const StepArgs<R> &a, int64_t p, int32_t k0, int32_t k1,
                                             const int32_t *nb, uint32_t *wp, const FBlock<R> &B, int tp,
                                             const FPair<R> &pp0, typename Tr<R>::V4 xp, typename Tr<R>::V4 up,
                                             R Ap, R Bp, R &fx, R &fy, R &fz) {
    using V4 = typename Tr<R>::V4;
    FPair<R> pp = pp0;
    const V4 nx{-xp.x, -xp.y, -xp.z, R(0)}, nu{-up.x, -up.y, -up.z, R(0)};
    const V4 *xb = a.xu + 2 * p;
    float2 fxy = make_float2(0.f, 0.f);
    // one slot: kinematics, stretch test, force term into the accumulators;
    // returns whether the bond stays within the critical stretch
    auto slot = [&](bool live, const V4 &xq, const V4 &uq, int32_t o) -> bool {
        const Kin<R> k(xq, uq, nx, nu);
        const R num = k.num, xx2 = k.xx2;
        const R wq = xq.w;
        const R lx = Tr<R>::sqrt_(xx2), ly = Tr<R>::sqrt_(xx2 + num);
        const R dl = Tr<R>::fma_(ly, lx, xx2);
        if (MULTI && live) pp = a.fp[B.pair_base + tp + (a.tinfo[p + o] & 255) * B.nt];
        const bool ok = num < pp.cs * dl;
        R tn;
        if (KIND == PD_MAT_BOND_BASED) {
            tn = num;
        } else {
            const typename Tr<R>::V2 mq = a.mab[p + o];
            tn = Tr<R>::fma_(pp.k35 * (Ap + mq.x), dl, pp.g15 * num * (Bp + mq.y));
        }
        const R coef = (live && ok) ? tn * wq * Tr<R>::rcp(dl * ly) : R(0);
        if constexpr (sizeof(R) == 4) k.accumulate(coef, fxy, fz);
        else k.accumulate(coef, fx, fy, fz);
        return ok;
    };
    for (int32_t w0 = k0, wend; w0 < k1; w0 = wend) {
        wend = min(k1, (w0 | 31) + 1);
        uint32_t *wptr = wp + 32 * (w0 >> 5);
        const int32_t kend = wend - w0;
        const uint32_t bits = range_bits(*wptr, w0, kend);
        if (!bits) continue;
        const int32_t *np = nb + w0;
        uint32_t okm = 0;
        int32_t o[U];
        load_offsets<U>(np, o);  // past the chunk: padded array, unused values
        int32_t j = 0;
        for (; j + U <= kend; j += U) {
            V4 xq[U], uq[U];
            int32_t oc[U];  // this group's offsets (state-based and multi-type terms read p + o)
#pragma unroll
            for (int u = 0; u < U; ++u) {
                Tr<R>::template load_rec<NC>(xb + 2 * (int64_t)o[u], xq[u], uq[u]);
                oc[u] = o[u];
            }
            // the next group's offsets, in flight while this group computes
            load_offsets<U>(np + j + U, o);
            const uint32_t bg = bits >> j;  // bit u <-> slot j + u
            uint32_t okg = 0;
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (slot((bg & (1u << u)) != 0u, xq[u], uq[u], oc[u])) okg |= 1u << u;
            okm |= okg << j;
        }
        // remaining kend - j < U slots; o[] holds their offsets
#pragma unroll
        for (int u = 0; u < U - 1; ++u) {
            if (j + u < kend) {
                V4 xq, uq;
                Tr<R>::template load_rec<NC>(xb + 2 * (int64_t)o[u], xq, uq);
                if (slot(((bits >> (j + u)) & 1u) != 0u, xq, uq, o[u])) okm |= 1u << (j + u);
            }
        }
        const uint32_t brk = bits & ~okm;
        if (kBreak && brk) atomicAnd(wptr, ~(brk << (w0 & 31)));
    }
    if constexpr (sizeof(R) == 4) {
        fx += fxy.x;
        fy += fxy.y;
    }
}

template <class R, int KIND, bool kBreak, int WPS, int U, bool NC = true, bool STG = false>
__device__ __forceinline__ void bond_gather(const StepArgs<R> &a, int64_t p, int w, const FBlock<R> &B, int tp,
                                            const FPair<R> &pp0, typename Tr<R>::V4 xp, typename Tr<R>::V4 up, const SliceInfo &d,
                                            int32_t cp, R &fx, R &fy, R &fz,
                                            const typename Tr<R>::V4 *stg = nullptr) {
    int32_t k0, k1;
    warp_range<WPS>(d.len, w, k0, k1);
    k1 = min(k1, cp);
    uint32_t *wp = a.words + d.word + (p & 31);
    R Ap = 0, Bp = 0, rtdp = 0;
    if (KIND != PD_MAT_BOND_BASED) {
        typename Tr<R>::V2 m = a.mab[p];
        Ap = m.x;
        Bp = m.y;
    }
    if (KIND == PD_MAT_ELASTO_PLASTIC) rtdp = a.rtd[p];
    if constexpr (STG) {
        if (stg) {  // a staged slice is a stencil slice
            const int32_t *sp = a.spos + d.nbr;
            if (B.nt > 1)
                bond_walk<R, KIND, kBreak, WPS, U, true, true, NC, true>(a, p, k0, k1, a.nbr + d.nbr, wp, B, tp, pp0, xp,
                                                                     up, Ap, Bp, fx, fy, fz, stg, sp);
            else
                bond_walk<R, KIND, kBreak, WPS, U, true, false, NC, true>(a, p, k0, k1, a.nbr + d.nbr, wp, B, tp, pp0, xp,
                                                                      up, Ap, Bp, fx, fy, fz, stg, sp);
            return;
        }
    }
    constexpr bool kAhead = KIND != PD_MAT_ELASTO_PLASTIC;  // stencil walks with offsets loaded ahead
    if (B.nt > 1) {
        if (kAhead && d.mode == kStencil)
            bond_walk_st<R, KIND, kBreak, U, true, NC>(a, p, k0, k1, a.nbr + d.nbr, wp, B, tp, pp0, xp, up, Ap, Bp, fx,
                                                       fy, fz);
        else if (d.mode == kStencil)
            bond_walk<R, KIND, kBreak, WPS, U, true, true, NC>(a, p, k0, k1, a.nbr + d.nbr, wp, B, tp, pp0, xp, up, Ap, Bp, fx,
                                                           fy, fz, nullptr, nullptr, rtdp);
        else
            bond_walk<R, KIND, kBreak, WPS, U, false, true, NC>(a, p, k0, k1, a.nbr + d.nbr + (p & 31), wp, B, tp, pp0, xp, up,
                                                            Ap, Bp, fx, fy, fz, nullptr, nullptr, rtdp);
    } else {
        if (kAhead && d.mode == kStencil)
            bond_walk_st<R, KIND, kBreak, U, false, NC>(a, p, k0, k1, a.nbr + d.nbr, wp, B, tp, pp0, xp, up, Ap, Bp, fx,
                                                        fy, fz);
        else if (d.mode == kStencil)
            bond_walk<R, KIND, kBreak, WPS, U, true, false, NC>(a, p, k0, k1, a.nbr + d.nbr, wp, B, tp, pp0, xp, up, Ap, Bp, fx,
                                                            fy, fz, nullptr, nullptr, rtdp);
        else
            bond_walk<R, KIND, kBreak, WPS, U, false, false, NC>(a, p, k0, k1, a.nbr + d.nbr + (p & 31), wp, B, tp, pp0, xp,
                                                             up, Ap, Bp, fx, fy, fz, nullptr, nullptr, rtdp);
    }
}

// BC velocity (boundary_conditions.jl:122-126): FixBC v = 0, ToFroBC v = dir*rate.
template <class R>
// Fix / ScaleFixWait / DeltaScale: v = 0; ToFro: v = dir*rate; Container
// (ContainerBC.jl:63-68): v = 0 once the current position left the limits.
__device__ __forceinline__ void bc_velocity(const StepArgs<R> &a, int64_t p, uint8_t bits, R &v0, R &v1, R &v2) {
    for (int k = 0; k < a.nbc; ++k) {
        if (!((bits >> k) & 1)) continue;
        const FBC &b = a.bc[k];
        const double dir = ((a.dir_vel >> k) & 1) ? -1.0 : 1.0;
        R vv[3] = {v0, v1, v2};
        if (b.kind == PD_BC_CONTAINER) {
            if (!b.has_limits) continue;
            double u0, u1, u2;
            load_u(a, p, u0, u1, u2);
            const double4 x = a.x64[p];
            const double y[3] = {x.x + u0, x.y + u1, x.z + u2};
            bool out = false;
            for (int d = 0; d < 3; ++d)
                if ((b.dims >> d) & 1) out |= (y[d] < b.lo[d]) || (y[d] > b.hi[d]);
            if (!out) continue;
            for (int d = 0; d < 3; ++d)
                if ((b.dims >> d) & 1) vv[d] = R(0);
        } else {
            for (int d = 0; d < 3; ++d)
                if ((b.dims >> d) & 1) vv[d] = b.kind == PD_BC_TOFRO ? R(dir * b.rate[d]) : R(0);
        }
        v0 = vv[0];
        v1 = vv[1];
        v2 = vv[2];
    }
}

// BC position (boundary_conditions.jl:107-111) on the FP64 displacement.
template <class R>
__device__ __forceinline__ void bc_position(const StepArgs<R> &a, int64_t p, uint8_t bits, double &u0, double &u1,
                                            double &u2) {
    const double4 x = a.x64[p];
    double y[3] = {x.x + u0, x.y + u1, x.z + u2};
    for (int k = 0; k < a.nbc; ++k) {
        if (!((bits >> k) & 1)) continue;
        const FBC &b = a.bc[k];
        if (b.kind == PD_BC_CONTAINER) continue;
        const int64_t r = b.rank[p - b.rank_lo];
        double4 last = b.last[r];
        const double step = a.dt * (((a.dir_pos >> k) & 1) ? -1.0 : 1.0);
        for (int d = 0; d < 3; ++d) {
            if (!((b.dims >> d) & 1)) continue;
            if (b.kind == PD_BC_FIX || b.kind == PD_BC_SCALE_FIX_WAIT) {
                y[d] = cmp(last, d);
            } else if (b.kind == PD_BC_DELTA_SCALE) {
                const double g = 1.0 + (b.scale[d] * a.dt) * (double)a.ts;
                y[d] = (cmp(last, d) - b.fix[d]) * g + b.fix[d];
            } else {
                const double nl = cmp(last, d) + step * b.rate[d];
                y[d] = nl;
                cmp(last, d) = nl;
            }
        }
        if (b.kind == PD_BC_TOFRO) b.last[r] = last;
    }
    u0 = y[0] - x.x;
    u1 = y[1] - x.y;
    u2 = y[2] - x.z;
}

template <class R>
__device__ __forceinline__ void load_u(const StepArgs<R> &a, int64_t p, double &u0, double &u1, double &u2) {
    if (sizeof(R) == 4) {
        u0 = a.ax[p];
        u1 = a.ay[p];
        u2 = a.az[p];
    } else {
        const typename Tr<R>::V4 u = a.xu[2 * p + 1];
        u0 = (double)u.x;
        u1 = (double)u.y;
        u2 = (double)u.z;
    }
}

template <class R>
__device__ __forceinline__ void store_u(const StepArgs<R> &a, int64_t p, double u0, double u1, double u2) {
    if (sizeof(R) == 4) {
        a.ax[p] = u0;
        a.ay[p] = u1;
        a.az[p] = u2;
    }
    typename Tr<R>::V4 o;
    o.x = (R)u0;
    o.y = (R)u1;
    o.z = (R)u2;
    o.w = a.xu[2 * p].w;  // the record weight, kept in both halves
    a.xn[2 * p + 1] = o;
}

// MODE 0: force only (update_acc!): f, p = m v.
// MODE 1: full step, another step follows: f, kick, BC vel, kick, drift,
//         BC pos -> next displacement.
// MODE 2: full step, last of the chunk: f, p, kick, BC vel, store v and f.
// MODE 3: integration only (forces already in f, e.g. after contacts).
// MODE 4: integration only, last of the chunk.
// MODE 5: force only into a scratch array, no bond breaking.
template <class R, int MODE>
__device__ __forceinline__ void integrate(const StepArgs<R> &a, int64_t p, R fx, R fy, R fz);

// Programmatic dependent launch.  The bond kernels are launched with
// programmatic stream serialization (launch_dep): a kernel's blocks may be
// dispatched while the previous kernel on the stream finishes, and wait
// here, before they read anything a previous kernel writes, until it has
// completed and its writes are visible.  Having passed the wait, a block lets the next
// kernel be dispatched in turn, so at most two grids of the chain are in
// flight and the older one never waits.  Without the launch attribute
// both instructions return at once.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// One step of one slice (its WPS warps): bond gather, fixed-order
// combination, integration.  Shared by k_step and the persistent kernel.
// PDL: the kernel was launched as a programmatic dependent (k_step); the
// data written only at initialisation (particle types, block and pair
// parameters, slice descriptors, slot counts) is read before pdl_enter,
// everything a previous kernel writes after it.  With all_def the gate
// flags are not read at all.
template <class R, int WPS, int U, int MODE, bool NC, bool STG = false, bool EPK = false, bool PDL = false>
__device__ __forceinline__ void step_body(const StepArgs<R> &a, int64_t blk, R (*sh)[3][32], int *arrive,
                                          const typename Tr<R>::V4 *stg = nullptr) {
    using V4 = typename Tr<R>::V4;
    constexpr int SPB = Split<WPS>::SPB;
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = wid % WPS;
    const int64_t p = (blk * SPB + wid / WPS) * 32 + lane;
    if (NC && p - lane < a.N) prefetch_slice_indices<WPS>(a.nbr, a.si, p >> 5, w, lane);
    const int32_t ti = p < a.N ? a.tinfo[p] : -1;
    constexpr bool kBreak = MODE != 5;
    R f[3] = {0, 0, 0};
    FBlock<R> B{};
    FPair<R> pp0{};
    SliceInfo d{};
    int32_t cp = 0;
    if (ti >= 0) {
        B = a.fb[ti >> 8];
        const int tp = ti & 255;
        if (B.kind != PD_MAT_SKIP) pp0 = a.fp[B.pair_base + tp + tp * B.nt];
        d = a.si[p >> 5];
        cp = a.cnt[p];
    }
    if (PDL) pdl_enter();
    if (ti >= 0) {
        const int b = ti >> 8, tp = ti & 255;
        if (B.kind != PD_MAT_SKIP && (a.all_def || a.deformed[b])) {
            V4 xp, up;
            Tr<R>::template load_rec<NC>(a.xu + 2 * p, xp, up);
            if (B.kind == PD_MAT_BOND_BASED) {
                bond_gather<R, PD_MAT_BOND_BASED, kBreak, WPS, U, NC, STG>(a, p, w, B, tp, pp0, xp, up, d, cp, f[0], f[1], f[2],
                                                                           stg);
            } else if (EPK && B.kind == PD_MAT_ELASTO_PLASTIC) {
                if constexpr (EPK)
                    bond_gather<R, PD_MAT_ELASTO_PLASTIC, kBreak, WPS, U, NC>(a, p, w, B, tp, pp0, xp, up, d, cp, f[0], f[1],
                                                                              f[2]);
            } else
                bond_gather<R, PD_MAT_ORDINARY_STATE_BASED, kBreak, WPS, U, NC, STG>(a, p, w, B, tp, pp0, xp, up, d, cp, f[0],
                                                                                     f[1], f[2], stg);
        }
    }
    if (WPS > 1 && !last_arrival_sum<WPS, 3>(sh, arrive, wid, lane, f)) return;
    const R fx = f[0], fy = f[1], fz = f[2];
    if (p >= a.N) return;
    if (ti < 0) {
        if (MODE == 1) a.xn[2 * p + 1] = V4{};
        return;
    }
    const R ir = a.irho[p];
    integrate<R, MODE>(a, p, fx * ir, fy * ir, fz * ir);
}

// Elasto-plastic kernels (EPK) keep more state per bond: up to 128 registers.
template <class R, int WPS, int U, int MODE, bool EPK = false>
__global__ void __launch_bounds__(Split<WPS>::BT, sizeof(R) != 4 ? 1
                                                  : EPK     ? Split<WPS>::MINB / 2
                                                  : U <= 2  ? Split<WPS>::MINB_U2
                                                            : Split<WPS>::MINB)
    k_step(StepArgs<R> a) {
    constexpr int NW = Split<WPS>::NW, SPB = Split<WPS>::SPB;
    __shared__ R sh[WPS > 1 ? NW : 1][3][32];
    __shared__ int arrive[SPB];
    if (WPS > 1) {
        if (threadIdx.x < SPB) arrive[threadIdx.x] = 0;
        __syncthreads();
    }
    step_body<R, WPS, U, MODE, true, false, EPK, true>(a, slice_of_block<SPB>(a), sh, arrive);
}

// MODE 3/4: integration of forces already in f (after contact forces).
template <class R, int MODE>
__global__ void __launch_bounds__(kT) k_integrate(StepArgs<R> a) {
    using V4 = typename Tr<R>::V4;
    const int64_t p = blockIdx.x * (int64_t)kT + threadIdx.x;
    if (p >= a.N) return;
    if (a.tinfo[p] < 0) {
        if (MODE == 3) a.xn[2 * p + 1] = V4{};
        return;
    }
    const V4 ff = a.f[p];
    integrate<R, MODE>(a, p, ff.x, ff.y, ff.z);
}

template <class R, int MODE>
__device__ __forceinline__ void integrate(const StepArgs<R> &a, int64_t p, R fx, R fy, R fz) {
    using V4 = typename Tr<R>::V4;
    if (MODE == 5) {
        a.f[p] = V4{fx, fy, fz, R(0)};
        return;
    }
    V4 vp = a.v[p];
    if (MODE == 0) {
        a.f[p] = V4{fx, fy, fz, R(0)};
        const R m = a.mass[p];
        a.p[p] = V4{m * vp.x, m * vp.y, m * vp.z, R(0)};
        return;
    }
    if (MODE == 2 || MODE == 4) {
        const R m = a.mass[p];
        if (MODE == 2) a.p[p] = V4{m * vp.x, m * vp.y, m * vp.z, R(0)};
    }
    if ((MODE == 1 || MODE == 2) && a.cacc) {
        const typename Tr<R>::V4 c = a.cacc[p];
        fx += c.x;
        fy += c.y;
        fz += c.z;
    }
    const uint8_t bits = a.nbc ? a.bcbits[p] : 0;
    R v0 = Tr<R>::fma_(a.c, fx, vp.x), v1 = Tr<R>::fma_(a.c, fy, vp.y), v2 = Tr<R>::fma_(a.c, fz, vp.z);
    if (bits) bc_velocity(a, p, bits, v0, v1, v2);
    if (MODE == 2 || MODE == 4) {
        a.v[p] = V4{v0, v1, v2, R(0)};
        a.f[p] = V4{fx, fy, fz, R(0)};
        return;
    }
    v0 = Tr<R>::fma_(a.c, fx, v0);
    v1 = Tr<R>::fma_(a.c, fy, v1);
    v2 = Tr<R>::fma_(a.c, fz, v2);
    double u0, u1, u2;
    load_u(a, p, u0, u1, u2);
    u0 = fma(a.dt, (double)v0, u0);
    u1 = fma(a.dt, (double)v1, u1);
    u2 = fma(a.dt, (double)v2, u2);
    if (bits) bc_position(a, p, bits, u0, u1, u2);
    a.v[p] = V4{v0, v1, v2, R(0)};
    store_u(a, p, u0, u1, u2);
}

// First half of a step (velocity_verlet.jl:62-69) from the stored force.
template <class R>
__device__ __forceinline__ void prologue_body(const StepArgs<R> &a, int64_t p) {
    using V4 = typename Tr<R>::V4;
    if (p >= a.N) return;
    if (a.tinfo[p] < 0) {
        a.xn[2 * p + 1] = V4{};
        return;
    }
    const V4 ff = a.f[p], vp = a.v[p];
    const R v0 = Tr<R>::fma_(a.c, ff.x, vp.x), v1 = Tr<R>::fma_(a.c, ff.y, vp.y), v2 = Tr<R>::fma_(a.c, ff.z, vp.z);
    double u0, u1, u2;
    load_u(a, p, u0, u1, u2);
    u0 = fma(a.dt, (double)v0, u0);
    u1 = fma(a.dt, (double)v1, u1);
    u2 = fma(a.dt, (double)v2, u2);
    const uint8_t bits = a.nbc ? a.bcbits[p] : 0;
    if (bits) bc_position(a, p, bits, u0, u1, u2);
    a.v[p] = V4{v0, v1, v2, R(0)};
    store_u(a, p, u0, u1, u2);
}

template <class R>
__global__ void __launch_bounds__(kT) k_prologue(StepArgs<R> a) {
    prologue_body(a, blockIdx.x * (int64_t)kT + threadIdx.x);
}

template <class R, int WPS, int U, bool ST, bool NC = true, bool STG = false>
__device__ __forceinline__ R theta_walk(const StepArgs<R> &a, int64_t p, int32_t k0, int32_t k1, const int32_t *nb,
                                        const uint32_t *wp, typename Tr<R>::V4 xp, typename Tr<R>::V4 up,
                                        const typename Tr<R>::V4 *stg = nullptr, const int32_t *sp = nullptr) {
    using V4 = typename Tr<R>::V4;
    R acc = 0;
    const V4 nx{-xp.x, -xp.y, -xp.z, R(0)}, nu{-up.x, -up.y, -up.z, R(0)};
    for (int32_t w0 = k0, wend; w0 < k1; w0 = wend) {
        wend = min(k1, (w0 | 31) + 1);
        const int32_t kend = wend - w0;
        const uint32_t bits = range_bits(wp[32 * (w0 >> 5)], w0, kend);
        if (!bits) continue;
        const int32_t *np = nb + (ST ? 1 : 32) * w0;
        const int32_t *spp = STG ? sp + w0 : nullptr;
        uint32_t bit = 1u;
#pragma unroll U
        for (int32_t j = 0; j < kend; ++j, bit <<= 1) {
            V4 xq, uq;
            if constexpr (STG) {
                const int32_t r = __ldg(spp + j) + (int32_t)(p & 31);
                xq = stg[2 * r];
                uq = stg[2 * r + 1];
            } else {
                const int32_t q = slot_neighbour<ST>(np, j, p);
                Tr<R>::template load_rec<NC>(a.xu + 2 * (int64_t)q, xq, uq);
            }
            const Kin<R> k(xq, uq, nx, nu);
            const R num = k.num;
            const R lx = Tr<R>::sqrt_(k.xx2), ly = Tr<R>::sqrt_(k.xx2 + num);
            const R term = num * xq.w * Tr<R>::rcp(ly + lx);
            acc += (bits & bit) ? term : R(0);
        }
    }
    return acc;
}

// theta_walk over a stencil slice with the slot offsets loaded one group of
// U slots ahead (as bond_walk_st); same terms in the same order.
template <class R, int U, bool NC>
__device__ __forceinline__ R theta_walk_st(const StepArgs<R> &a, int64_t p, int32_t k0, int32_t k1,
                                           const int32_t *nb, const uint32_t *wp, typename Tr<R>::V4 xp,
                                           typename Tr<R>::V4 up) {
    using V4 = typename Tr<R>::V4;
    R acc = 0;
    const V4 nx{-xp.x, -xp.y, -xp.z, R(0)}, nu{-up.x, -up.y, -up.z, R(0)};
    const V4 *xb = a.xu + 2 * p;
    auto term = [&](const V4 &xq, const V4 &uq, bool live) {
        const Kin<R> k(xq, uq, nx, nu);
        const R num = k.num;
        const R lx = Tr<R>::sqrt_(k.xx2), ly = Tr<R>::sqrt_(k.xx2 + num);
        const R t = num * xq.w * Tr<R>::rcp(ly + lx);
        acc += live ? t : R(0);
    };
    for (int32_t w0 = k0, wend; w0 < k1; w0 = wend) {
        wend = min(k1, (w0 | 31) + 1);
        const int32_t kend = wend - w0;
        const uint32_t bits = range_bits(wp[32 * (w0 >> 5)], w0, kend);
        if (!bits) continue;
        const int32_t *np = nb + w0;
        int32_t o[U];
        load_offsets<U>(np, o);  // past the chunk: padded array, unused values
        int32_t j = 0;
        for (; j + U <= kend; j += U) {
            V4 xq[U], uq[U];
#pragma unroll
            for (int u = 0; u < U; ++u) Tr<R>::template load_rec<NC>(xb + 2 * (int64_t)o[u], xq[u], uq[u]);
            load_offsets<U>(np + j + U, o);
            const uint32_t bg = bits >> j;
#pragma unroll
            for (int u = 0; u < U; ++u) term(xq[u], uq[u], (bg & (1u << u)) != 0u);
        }
#pragma unroll
        for (int u = 0; u < U - 1; ++u) {
            if (j + u < kend) {
                V4 xq, uq;
                Tr<R>::template load_rec<NC>(xb + 2 * (int64_t)o[u], xq, uq);
                term(xq, uq, (bits >> (j + u)) & 1u);
            }
        }
    }
    return acc;
}

// Dilatation (peri.jl:155-172): theta_p = 3/m_p sum_q e_pq V_q over intact
// bonds; stores theta_p/m_p for the force pass.  Same warp split as k_step.
template <class R, int WPS, int U, bool NC, bool STG = false, bool PDL = false>
__device__ __forceinline__ void theta_body(const StepArgs<R> &a, int64_t blk, R (*sh)[1][32], int *arrive,
                                           const typename Tr<R>::V4 *stg = nullptr) {
    using V4 = typename Tr<R>::V4;
    constexpr int SPB = Split<WPS>::SPB;
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = wid % WPS;
    const int64_t p = (blk * SPB + wid / WPS) * 32 + lane;
    if (NC && p - lane < a.N) prefetch_slice_indices<WPS>(a.nbr, a.si, p >> 5, w, lane);
    const int32_t ti = p < a.N ? a.tinfo[p] : -1;
    const bool lps = ti >= 0 && (a.fb[ti >> 8].kind == PD_MAT_ORDINARY_STATE_BASED ||
                                 a.fb[ti >> 8].kind == PD_MAT_ELASTO_PLASTIC);
    SliceInfo d{};
    int32_t cp = 0;
    if (lps) {
        d = a.si[p >> 5];
        cp = a.cnt[p];
    }
    if (PDL) pdl_enter();
    R acc = 0;
    if (lps) {
        V4 xp, up;
        Tr<R>::template load_rec<NC>(a.xu + 2 * p, xp, up);
        int32_t k0, k1;
        warp_range<WPS>(d.len, w, k0, k1);
        k1 = min(k1, cp);
        const uint32_t *wp = a.words + d.word + (p & 31);
        if (STG && stg)
            acc = theta_walk<R, WPS, U, true, NC, true>(a, p, k0, k1, a.nbr + d.nbr, wp, xp, up, stg,
                                                        a.spos + d.nbr);
        else if (d.mode == kStencil)
            acc = theta_walk_st<R, U, NC>(a, p, k0, k1, a.nbr + d.nbr, wp, xp, up);
        else
            acc = theta_walk<R, WPS, U, false, NC>(a, p, k0, k1, a.nbr + d.nbr + (p & 31), wp, xp, up);
    }
    if (WPS > 1 && !last_arrival_sum<WPS, 1>(sh, arrive, wid, lane, &acc)) return;
    if (!lps) return;
    typename Tr<R>::V2 mb = a.mab[p];
    mb.x = R(3) * acc * mb.y * mb.y;  // theta/m = (3/m) acc / m
    a.mab[p] = mb;
}

template <class R, int WPS, int U>
__global__ void __launch_bounds__(Split<WPS>::BT, sizeof(R) == 4 ? Split<WPS>::MINB_THETA : 1) k_theta(StepArgs<R> a) {
    constexpr int NW = Split<WPS>::NW, SPB = Split<WPS>::SPB;
    __shared__ R sh[WPS > 1 ? NW : 1][1][32];
    __shared__ int arrive[SPB];
    if (WPS > 1) {
        if (threadIdx.x < SPB) arrive[threadIdx.x] = 0;
        __syncthreads();
    }
    theta_body<R, WPS, U, true, false, true>(a, slice_of_block<SPB>(a), sh, arrive);
}

// ---------------------------------------------------------------------
// Job-table kernels of the serving loop: one launch advances up to
// kJobsPerLaunch resident jobs of a batch (separate environments, each with
// its own buffers, time step and parameters).  The table is the launch's
// parameter (t.a[j]: job j's step arguments, t.bstart[j]: its first block,
// t.bstart[n] the grid size), read in place from the parameter bank
// (__grid_constant__), so the job's arguments cost no registers, as in the
// single-environment kernels.  A block finds its job by a binary search
// over t.bstart and runs the same body as the single-environment kernel
// over its own slices, so a job computes the same numbers in a batch as
// alone.
// ---------------------------------------------------------------------
constexpr int kJobsPerLaunch = 16;  // 16 x 1856-byte arguments: within the 32 KB parameter limit
template <class R>
struct JobTable {
    StepArgs<R> a[kJobsPerLaunch];
    int32_t bstart[kJobsPerLaunch + 1];
    int32_t n;
};
static_assert(sizeof(JobTable<float>) <= 32764 && sizeof(JobTable<double>) <= 32764,
              "a job table must fit the kernel parameter space");

template <class R>
__device__ __forceinline__ int job_of_block(const JobTable<R> &t, int32_t b) {
    int lo = 0, hi = t.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t.bstart[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <class R, int WPS, int U, int MODE>
__global__ void __launch_bounds__(Split<WPS>::BT, sizeof(R) != 4 ? 1 : U <= 2 ? Split<WPS>::MINB_U2 : Split<WPS>::MINB)
    k_step_jobs(const __grid_constant__ JobTable<R> t) {
    constexpr int NW = Split<WPS>::NW, SPB = Split<WPS>::SPB;
    __shared__ R sh[WPS > 1 ? NW : 1][3][32];
    __shared__ int arrive[SPB];
    if (WPS > 1) {
        if (threadIdx.x < SPB) arrive[threadIdx.x] = 0;
        __syncthreads();
    }
    const int j = job_of_block(t, (int32_t)blockIdx.x);
    step_body<R, WPS, U, MODE, true>(t.a[j], (int32_t)blockIdx.x - t.bstart[j], sh, arrive);
}

template <class R, int WPS, int U>
__global__ void __launch_bounds__(Split<WPS>::BT, sizeof(R) == 4 ? Split<WPS>::MINB_THETA : 1)
    k_theta_jobs(const __grid_constant__ JobTable<R> t) {
    constexpr int NW = Split<WPS>::NW, SPB = Split<WPS>::SPB;
    __shared__ R sh[WPS > 1 ? NW : 1][1][32];
    __shared__ int arrive[SPB];
    if (WPS > 1) {
        if (threadIdx.x < SPB) arrive[threadIdx.x] = 0;
        __syncthreads();
    }
    const int j = job_of_block(t, (int32_t)blockIdx.x);
    theta_body<R, WPS, U, true>(t.a[j], (int32_t)blockIdx.x - t.bstart[j], sh, arrive);
}

template <class R>
__global__ void __launch_bounds__(kT) k_prologue_jobs(const __grid_constant__ JobTable<R> t) {
    const int j = job_of_block(t, (int32_t)blockIdx.x);
    prologue_body(t.a[j], ((int32_t)blockIdx.x - t.bstart[j]) * (int64_t)kT + threadIdx.x);
}

// ---------------------------------------------------------------------
// Elasto-plastic td_norm2 pass (elasto_plastic.jl:274-288 through
// loop_over_neighs!, peri.jl:411-445): td_norm2_p = sum over intact bonds
// within the critical stretch of td_trial^2 V_q, with p's own plastic
// strain; bonds at or beyond the critical stretch break here (the force
// walk that follows finds none).  The sum runs in FP64 in both precisions
// (td_trial^2 exceeds the FP32 range in SI units); stored as
// 1/sqrt(td_norm2) in the working precision.
// ---------------------------------------------------------------------
template <class R, int U, bool ST, bool MULTI>
__device__ __forceinline__ double td_walk(const StepArgs<R> &a, int64_t p, int32_t k0, int32_t k1,
                                          const int32_t *nb, uint32_t *wp, const FBlock<R> &B, int tp,
                                          typename Tr<R>::V4 xp, typename Tr<R>::V4 up, R Ap, R Bp) {
    using V4 = typename Tr<R>::V4;
    FPair<R> pp = a.fp[B.pair_base + tp + tp * B.nt];
    const V4 nx{-xp.x, -xp.y, -xp.z, R(0)}, nu{-up.x, -up.y, -up.z, R(0)};
    double acc = 0.0;
    for (int32_t w0 = k0, wend; w0 < k1; w0 = wend) {
        wend = min(k1, (w0 | 31) + 1);
        uint32_t *wptr = wp + 32 * (w0 >> 5);
        const int32_t kend = wend - w0;
        const uint32_t bits = range_bits(*wptr, w0, kend);
        if (!bits) continue;
        const int32_t *np = nb + (ST ? 1 : 32) * w0;
        const int64_t ebase = ((int64_t)(wptr - a.words) << 5) + (w0 & 31);
        uint32_t okm = 0, bit = 1u;
#pragma unroll U
        for (int32_t j = 0; j < kend; ++j, bit <<= 1) {
            const int32_t q = slot_neighbour<ST>(np, j, p);
            V4 xq, uq;
            Tr<R>::template load_rec<true>(a.xu + 2 * (int64_t)q, xq, uq);
            const Kin<R> k(xq, uq, nx, nu);
            const R num = k.num, xx2 = k.xx2;
            const R lx = Tr<R>::sqrt_(xx2), ly = Tr<R>::sqrt_(xx2 + num);
            const R dl = Tr<R>::fma_(ly, lx, xx2);
            const bool live = (bits & bit) != 0u;
            if (MULTI && live) pp = a.fp[B.pair_base + tp + (a.tinfo[q] & 255) * B.nt];
            const bool ok = num < pp.cs * dl;
            okm |= ok ? bit : 0u;
            const typename Tr<R>::V2 mq = a.mab[q];
            const R As = Ap + mq.x, Bs = Bp + mq.y;
            const R ed = Tr<R>::fma_(-As * Tr<R>::rcp(Bs), lx * R(1.0 / 3.0), num * Tr<R>::rcp(ly + lx));
            const R tdt = pp.g15 * Tr<R>::rcp(lx) * Bs * (ed - (R)a.edp_in[ebase + j]);
            const double t2 = (double)tdt * (double)tdt * (double)xq.w;
            acc += (live && ok) ? t2 : 0.0;
        }
        const uint32_t brk = bits & ~okm;
        if (brk) atomicAnd(wptr, ~(brk << (w0 & 31)));
    }
    return acc;
}

template <class R, int WPS, int U>
__device__ __forceinline__ void td_body(const StepArgs<R> &a, int64_t blk, double (*sh)[1][32], int *arrive) {
    using V4 = typename Tr<R>::V4;
    constexpr int SPB = Split<WPS>::SPB;
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = wid % WPS;
    const int64_t p = (blk * SPB + wid / WPS) * 32 + lane;
    const int32_t ti = p < a.N ? a.tinfo[p] : -1;
    // data written only at initialisation before the dependent-launch wait
    FBlock<R> B{};
    SliceInfo d{};
    int32_t cp = 0;
    if (ti >= 0) {
        B = a.fb[ti >> 8];
        d = a.si[p >> 5];
        cp = a.cnt[p];
    }
    pdl_enter();
    const bool ep = ti >= 0 && B.kind == PD_MAT_ELASTO_PLASTIC && (a.all_def || a.deformed[ti >> 8]);
    double acc = 0.0;
    if (ep) {
        const int tp = ti & 255;
        V4 xp, up;
        Tr<R>::template load_rec<true>(a.xu + 2 * p, xp, up);
        int32_t k0, k1;
        warp_range<WPS>(d.len, w, k0, k1);
        k1 = min(k1, cp);
        uint32_t *wp = a.words + d.word + (p & 31);
        const typename Tr<R>::V2 m = a.mab[p];
        const bool st = d.mode == kStencil;
        const int32_t *nb = a.nbr + d.nbr + (st ? 0 : (p & 31));
        if (B.nt > 1) {
            acc = st ? td_walk<R, U, true, true>(a, p, k0, k1, nb, wp, B, tp, xp, up, m.x, m.y)
                     : td_walk<R, U, false, true>(a, p, k0, k1, nb, wp, B, tp, xp, up, m.x, m.y);
        } else {
            acc = st ? td_walk<R, U, true, false>(a, p, k0, k1, nb, wp, B, tp, xp, up, m.x, m.y)
                     : td_walk<R, U, false, false>(a, p, k0, k1, nb, wp, B, tp, xp, up, m.x, m.y);
        }
    }
    if (WPS > 1 && !last_arrival_sum<WPS, 1>(sh, arrive, wid, lane, &acc)) return;
    if (!ep) return;
    a.rtd[p] = acc > 0.0 ? (R)(1.0 / sqrt(acc)) : (R)INFINITY;
}

template <class R, int WPS, int U>
__global__ void __launch_bounds__(Split<WPS>::BT, Split<WPS>::MINB / 2) k_td(StepArgs<R> a) {
    constexpr int NW = Split<WPS>::NW, SPB = Split<WPS>::SPB;
    __shared__ double sh[WPS > 1 ? NW : 1][1][32];
    __shared__ int arrive[SPB];
    if (WPS > 1) {
        if (threadIdx.x < SPB) arrive[threadIdx.x] = 0;
        __syncthreads();
    }
    td_body<R, WPS, U>(a, slice_of_block<SPB>(a), sh, arrive);
}

// Per bond slot e of an elasto-plastic particle, the slot of the reverse
// bond in the neighbour's family (partner[e]); other slots point at
// themselves so that every read stays in range.
template <class R>
__global__ void __launch_bounds__(kT) k_partner(StepArgs<R> a, const uint32_t *fam, int32_t *partner) {
    const int64_t p = blockIdx.x * (int64_t)kT + threadIdx.x;
    if (p >= a.N) return;
    const SliceInfo d = a.si[p >> 5];
    const int32_t n = a.cnt[p];
    const int32_t ti = a.tinfo[p];
    const bool ep = ti >= 0 && a.fb[ti >> 8].kind == PD_MAT_ELASTO_PLASTIC;
    const bool st = d.mode == kStencil;
    const int32_t *nb = a.nbr + d.nbr + (st ? 0 : (p & 31));
    for (int32_t k = 0; k < d.len; ++k) {
        const int64_t e = slot_index(a.si, p, k);
        const bool member = ep && k < n && ((fam[e >> 5] >> (k & 31)) & 1u);
        if (!member) {
            partner[e] = (int32_t)e;
            continue;
        }
        const int32_t q = st ? (int32_t)p + nb[k] : nb[32 * k];
        const int32_t kq = slot_of(a.si, a.nbr, a.cnt, q, p);
        const SliceInfo dq = a.si[q >> 5];
        const bool found = kq < a.cnt[q] && (dq.mode == kStencil ? (int64_t)q + a.nbr[dq.nbr + kq] == p
                                                                 : a.nbr[dq.nbr + (q & 31) + 32 * (int64_t)kq] == p);
        partner[e] = found ? (int32_t)slot_index(a.si, q, kq) : (int32_t)e;
    }
}

// ---------------------------------------------------------------------
// Staged kernels (FP32C, 4 or 8 warps per slice, one slice per block).
// The neighbour records of a stencil slice are a few ranges of
// consecutive records (the 32-record windows of its offsets, merged); one
// thread copies them into shared memory with bulk asynchronous copies that
// complete on an mbarrier, and the walks then read shared memory instead
// of waiting on L1/L2 one slot at a time.  Same arithmetic and order as the
// global-load kernels, so the results are identical.
// ---------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

constexpr uint32_t kStageSpins = 1u << 22;  // bounded wait on the staging copies

// Returns the staged records of slice s in shared memory, or nullptr when
// the slice has no plan (its walks load from global memory) or when the
// copies did not complete within kStageSpins polls (error flag set; the
// block falls back to global loads).  Called by every thread of the block.
__device__ __forceinline__ const float4 *stage_slice(const StepArgs<float> &a, int64_t s, float4 *srec,
                                                     uint64_t *bar) {
    const int32_t so = a.splan_off[s];
    if (so < 0) return nullptr;
    const int32_t nr = a.splan[so], T = a.splan[so + 1];
    const uint32_t b = smem_u32(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"((uint32_t)T * 32u)
                     : "memory");
        int32_t base = 0;
        for (int32_t m = 0; m < nr; ++m) {
            const int32_t r0 = a.splan[so + 2 + 2 * m], len = a.splan[so + 3 + 2 * m];
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_u32(srec + 2 * base)),
                "l"(a.xu + 2 * (int64_t)r0), "r"((uint32_t)len * 32u), "r"(b)
                : "memory");
            base += len;
        }
    }
    for (uint32_t it = 0; it < kStageSpins; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], 0;\n selp.u32 %0, 1, 0, P;\n}"
            : "=r"(done)
            : "r"(b)
            : "memory");
        if (done) return srec;
    }
    if (threadIdx.x == 0) atomicExch(a.serr, 1);
    return nullptr;
}

template <int WPS, int U, int MODE>
__global__ void __launch_bounds__(Split<WPS>::BT, Split<WPS>::MINB) k_step_st(StepArgs<float> a) {
    static_assert(Split<WPS>::SPB == 1, "one slice per block");
    extern __shared__ __align__(128) float4 srec[];
    __shared__ float sh[WPS][3][32];
    __shared__ int arrive[1];
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) arrive[0] = 0;
    const float4 *stg = stage_slice(a, blockIdx.x, srec, &bar);
    __syncthreads();
    step_body<float, WPS, U, MODE, true, true>(a, blockIdx.x, sh, arrive, stg);
}

template <int WPS, int U>
__global__ void __launch_bounds__(Split<WPS>::BT, Split<WPS>::MINB_THETA) k_theta_st(StepArgs<float> a) {
    static_assert(Split<WPS>::SPB == 1, "one slice per block");
    extern __shared__ __align__(128) float4 srec[];
    __shared__ float sh[WPS][1][32];
    __shared__ int arrive[1];
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) arrive[0] = 0;
    const float4 *stg = stage_slice(a, blockIdx.x, srec, &bar);
    __syncthreads();
    theta_body<float, WPS, U, true, true>(a, blockIdx.x, sh, arrive, stg);
}

// ---------------------------------------------------------------------
// Persistent chunk: nsteps full steps (dilatation phase, force + integration
// phase) in one cooperative launch, phases separated by a grid barrier, so
// small problems pay no per-kernel launch and ramp-up.  Records written in
// one phase are read by other blocks in the next, hence coherent loads.
// ---------------------------------------------------------------------
struct GridBar {
    unsigned count, gen;
    int err, pad;
};
constexpr unsigned kBarrierSpins = 1u << 25;  // x >= 64 ns: gives up after ~2 s

// Grid-wide barrier of a cooperative launch; false (and the error flag set)
// when a block waited past kBarrierSpins.
__device__ __forceinline__ bool grid_barrier(GridBar *gb, unsigned nblocks) {
    __shared__ int ok;  // thread 0's reading of the error flag, so the whole block leaves together
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = &gb->gen;
        volatile int *verr = &gb->err;
        const unsigned g = *vgen;
        __threadfence();
        if (atomicAdd(&gb->count, 1u) == nblocks - 1) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            for (unsigned it = 0; *vgen == g && !*verr; ++it) {
                if (it > kBarrierSpins) {
                    atomicExch(&gb->err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok = *verr == 0;
    }
    __syncthreads();
    __threadfence();
    return ok != 0;
}

// The grid is at most what the device holds at once; each block walks the
// slice groups blockIdx.x, blockIdx.x + gridDim.x, ... of every phase (a
// block synchronises between groups when its warps share a slice, so the
// partial sums of one group are read before the next group writes them).
//
// The step arguments come as two read-only kernel parameters, one per
// record-buffer parity (a0: even steps read b0 and write b1; a1: the
// reverse), and are never modified: the walks then read every field from
// the parameter bank, as k_step does, instead of from a per-thread copy of
// the 1.8 KB structure in local memory.  The time step stays at the
// launch's value: persistent runs, like graph replays, carry no
// time-dependent boundary condition.
template <class R, int WPS, int U, bool LPS>
__device__ __forceinline__ bool persist_step(const StepArgs<R> &a, int64_t ngroups, GridBar *gb, R (*sh)[3][32],
                                             R (*sh1)[1][32], int *arrive) {
    if (LPS) {
        for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
            theta_body<R, WPS, U, false>(a, g, sh1, arrive);
            if (WPS > 1) __syncthreads();
        }
        if (!grid_barrier(gb, gridDim.x)) return false;
    }
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        step_body<R, WPS, U, 1, false>(a, g, sh, arrive);
        if (WPS > 1) __syncthreads();
    }
    return true;
}

template <class R, int WPS, int U, bool LPS>
__global__ void __launch_bounds__(Split<WPS>::BT, sizeof(R) == 4 ? Split<WPS>::MINB : 1)
    k_persist(const __grid_constant__ StepArgs<R> a0, const __grid_constant__ StepArgs<R> a1, int nsteps,
              GridBar *gb, int64_t ngroups) {
    constexpr int NW = Split<WPS>::NW, SPB = Split<WPS>::SPB;
    __shared__ R sh[WPS > 1 ? NW : 1][3][32];
    __shared__ R sh1[WPS > 1 ? NW : 1][1][32];
    __shared__ int arrive[SPB];
    if (WPS > 1) {
        if (threadIdx.x < SPB) arrive[threadIdx.x] = 0;
        __syncthreads();
    }
    for (int s = 0; s < nsteps; ++s) {
        const bool ok = (s & 1) ? persist_step<R, WPS, U, LPS>(a1, ngroups, gb, sh, sh1, arrive)
                                : persist_step<R, WPS, U, LPS>(a0, ngroups, gb, sh, sh1, arrive);
        if (!ok) return;
        if (s + 1 < nsteps && !grid_barrier(gb, gridDim.x)) return;
    }
}

// Deformed gate on y = x + u (general_material.jl:243-255).  kGB: the
// largest number of CTAs sharing one block's partial norms -- a fixed width
// rather than the device's SM count, so the norms' summation order does not
// depend on the GPU.
constexpr int kGB = 148, kGT = 256;
// One GateItem per block still undeformed; grid.y walks the list and
// grid.x = gx CTAs share each block, so any number of blocks is tested in
// two launches.
template <class R>
__global__ void __launch_bounds__(kGT) k_fgate_partial(StepArgs<R> a, const GateItem *items, int gx, double *part) {
    const GateItem it = items[blockIdx.y];
    double *out = part + 3 * ((int64_t)blockIdx.y * gx + blockIdx.x);
    if (a.deformed[it.block]) return;
    const int64_t first = it.first, n = it.n;
    __shared__ double sh[3][kGT];
    double u0, u1, u2;
    load_u(a, first, u0, u1, u2);
    const double4 x1 = a.x64[first];
    const double y10 = x1.x + u0, y11 = x1.y + u1, y12 = x1.z + u2;
    double sd = 0, sa = 0, sx = 0;
    for (int64_t l = blockIdx.x * (int64_t)kGT + threadIdx.x; l < n; l += (int64_t)gx * kGT) {
        const double4 xi = a.x64[first + l];
        load_u(a, first + l, u0, u1, u2);
        const double A0 = ((xi.x + u0) - y10) + x1.x, A1 = ((xi.y + u1) - y11) + x1.y, A2 = ((xi.z + u2) - y12) + x1.z;
        const double d0 = A0 - xi.x, d1 = A1 - xi.y, d2 = A2 - xi.z;
        sd += d0 * d0 + d1 * d1 + d2 * d2;
        sa += A0 * A0 + A1 * A1 + A2 * A2;
        sx += xi.x * xi.x + xi.y * xi.y + xi.z * xi.z;
    }
    sh[0][threadIdx.x] = sd;
    sh[1][threadIdx.x] = sa;
    sh[2][threadIdx.x] = sx;
    __syncthreads();
    for (int s = kGT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; ++c) out[c] = sh[c][0];
}

__global__ void k_fgate_final(const GateItem *items, int nitems, int gx, const double *part, int32_t *deformed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nitems) return;
    int32_t *flag = deformed + items[i].block;
    if (*flag) return;
    double sd = 0, sa = 0, sx = 0;
    for (int b = 0; b < gx; ++b) {
        const double *q = part + 3 * ((int64_t)i * gx + b);
        sd += q[0];
        sa += q[1];
        sx += q[2];
    }
    const double d = sqrt(sd);
    const bool approx = isfinite(d) && d <= fmax(0.0, 0x1p-26 * fmax(sqrt(sa), sqrt(sx)));
    if (!approx) *flag = 1;
}

// FP64 state -> fast state.
template <class R>
__global__ void k_import(int64_t N, const double4 *x4, const double4 *y, const double4 *v, const double4 *f,
                         const double4 *pm, const double *mass, const double *dens, const double2 *mth,
                         const int32_t *tinfo, const DevBlock *blocks, StepArgs<R> a) {
    using V4 = typename Tr<R>::V4;
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= N) return;
    const double4 xi = x4[p], yi = y[p], vi = v[p], fi = f[p], pi = pm[p];
    const double u0 = yi.x - xi.x, u1 = yi.y - xi.y, u2 = yi.z - xi.z;
    V4 xs;
    const int32_t ti = tinfo[p];
    // w: the volume, times the bond constant c in bond-based blocks (the
    // bond walk then needs no per-bond multiply by c)
    const double wv = (ti >= 0 && blocks[ti >> 8].kind == PD_MAT_BOND_BASED) ? blocks[ti >> 8].c11 * xi.w : xi.w;
    if (sizeof(R) == 4 && ti >= 0) {
        const double3 c = blocks[ti >> 8].center;
        xs = V4{(R)(xi.x - c.x), (R)(xi.y - c.y), (R)(xi.z - c.z), (R)wv};
    } else {
        xs = V4{(R)xi.x, (R)xi.y, (R)xi.z, (R)wv};
    }
    if (sizeof(R) == 4) {
        a.ax[p] = u0;
        a.ay[p] = u1;
        a.az[p] = u2;
    }
    // the reference position lives in both halves of the double buffer
    V4 *cur = const_cast<V4 *>(a.xu);
    cur[2 * p] = xs;
    a.xn[2 * p] = xs;
    cur[2 * p + 1] = V4{(R)u0, (R)u1, (R)u2, xs.w};
    a.xn[2 * p + 1] = V4{(R)u0, (R)u1, (R)u2, xs.w};
    a.v[p] = V4{(R)vi.x, (R)vi.y, (R)vi.z, R(0)};
    a.f[p] = V4{(R)fi.x, (R)fi.y, (R)fi.z, R(0)};
    a.p[p] = V4{(R)pi.x, (R)pi.y, (R)pi.z, R(0)};
    const_cast<R *>(a.irho)[p] = ti >= 0 ? (R)(1.0 / dens[p]) : R(0);
    const_cast<R *>(a.mass)[p] = (R)mass[p];
    const double m = mth[p].x;
    a.mab[p] = typename Tr<R>::V2{(R)(m > 0 ? mth[p].y / m : 0.0), (R)(m > 0 ? 1.0 / m : 0.0)};
}

// fast state -> FP64 state (y = x + u, v, f, p, theta).
template <class R>
__global__ void k_export(int64_t N, const double4 *x4, double4 *y, double4 *v, double4 *f, double4 *pm, double2 *mth,
                         StepArgs<R> a) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= N) return;
    double u0, u1, u2;
    load_u(a, p, u0, u1, u2);
    const double4 xi = x4[p];
    y[p] = make_double4(xi.x + u0, xi.y + u1, xi.z + u2, 0.0);
    const typename Tr<R>::V4 vi = a.v[p], fi = a.f[p], pi = a.p[p];
    v[p] = make_double4(vi.x, vi.y, vi.z, 0.0);
    f[p] = make_double4(fi.x, fi.y, fi.z, 0.0);
    pm[p] = make_double4(pi.x, pi.y, pi.z, 0.0);
    const typename Tr<R>::V2 mb = a.mab[p];
    if (mb.y != R(0)) mth[p].y = (double)mb.x / (double)mb.y;
}

// Contact accelerations added to the fast force (nonlinearspring.jl:124-145,
// contacts.jl:210-247 / 357-381), evaluated in FP64 on y = x + u.
struct CLawF {
    double equi, expo, K;
};
__device__ __forceinline__ void cfn(const CLawF &c, double d0, double d1, double d2, double &F0, double &F1,
                                    double &F2) {
    const double mag = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    const double del = c.equi - mag;
    if (del < 0.0) {
        F0 = F1 = F2 = 0.0;
        return;
    }
    const double strain = del / c.equi;
    double pw;
    if (c.expo == 1.0) pw = strain;
    else if (c.expo == 2.0) pw = strain * strain;
    else pw = pow(strain, c.expo);
    const double s = c.K * pw / (mag + 1e-10);
    F0 = s * d0;
    F1 = s * d1;
    F2 = s * d2;
}

template <class R>
__device__ __forceinline__ void ypos(const StepArgs<R> &a, int64_t p, double &y0, double &y1, double &y2) {
    double u0, u1, u2;
    load_u(a, p, u0, u1, u2);
    const double4 x = a.x64[p];
    y0 = x.x + u0;
    y1 = x.y + u1;
    y2 = x.z + u2;
}

// Sum of the 32 lanes' partial sums in a fixed butterfly order (every lane
// ends with the same bits: each stage adds the same two values).
__device__ __forceinline__ void warp_sum3(double &a0, double &a1, double &a2) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
}

template <class R>
__device__ __forceinline__ void add_contact(const StepArgs<R> &a, int64_t p, double a0, double a1, double a2) {
    typename Tr<R>::V4 f = a.f[p];
    f.x += (R)a0;
    f.y += (R)a1;
    f.z += (R)a2;
    a.f[p] = f;
}

// The contact kernels run over the lists of particles with contact work
// (act, nact entries; built with the neighbour lists), or over the whole
// set when act is null: one warp per listed particle, its lanes taking
// every 32nd neighbour row, the lanes' sums combined in a fixed order, so
// results do not depend on scheduling.  (A thread per particle left the
// few thousand listed particles of an impact to a handful of warps, each
// walking its rows one dependent load after another.)
template <class R>
__global__ void k_fc12_1(StepArgs<R> a, int64_t first1, int64_t n1, int64_t rows, const int32_t *nb,
                         const double *dens, CLawF law, const int32_t *act, int64_t nact) {
    const int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= nact) return;  // whole warps
    const int64_t i = act ? act[t] : t;
    const int64_t p = first1 + i;
    double yi0, yi1, yi2, a0 = 0, a1 = 0, a2 = 0;
    ypos(a, p, yi0, yi1, yi2);
    const double inv = 1.0 / dens[p];
    for (int64_t r0 = 0; r0 < rows; r0 += 32) {
        const int64_t r = r0 + lane;
        const int32_t j = r < rows ? nb[r * n1 + i] : -1;
        // a particle's rows end at the first -1; nothing past it is read
        const uint32_t stop = __ballot_sync(0xffffffffu, j < 0);
        const int nlive = stop ? __ffs(stop) - 1 : 32;
        if (lane < nlive) {
            double yj0, yj1, yj2, F0, F1, F2;
            ypos(a, j, yj0, yj1, yj2);
            cfn(law, yi0 - yj0, yi1 - yj1, yi2 - yj2, F0, F1, F2);
            const double s = a.x64[j].w * inv;
            a0 += F0 * s;
            a1 += F1 * s;
            a2 += F2 * s;
        }
        if (stop) break;
    }
    warp_sum3(a0, a1, a2);
    if (lane == 0) add_contact(a, p, a0, a1, a2);
}

template <class R>
__global__ void k_fc12_2(StepArgs<R> a, int64_t first2, int64_t n2, const int32_t *roff, const int32_t *rev,
                         const double *dens, CLawF law, const int32_t *act, int64_t nact) {
    const int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= nact) return;
    const int64_t j = act ? act[t] : t;
    const int32_t o = roff[j], e = roff[j + 1];
    if (o == e) return;
    const int64_t q = first2 + j;
    double yj0, yj1, yj2, a0 = 0, a1 = 0, a2 = 0;
    ypos(a, q, yj0, yj1, yj2);
    const double inv = 1.0 / dens[q];
    for (int32_t r = o + lane; r < e; r += 32) {
        const int32_t i = rev[r];
        double yi0, yi1, yi2, F0, F1, F2;
        ypos(a, i, yi0, yi1, yi2);
        cfn(law, yi0 - yj0, yi1 - yj1, yi2 - yj2, F0, F1, F2);
        const double s = a.x64[i].w * inv;
        a0 -= F0 * s;
        a1 -= F1 * s;
        a2 -= F2 * s;
    }
    warp_sum3(a0, a1, a2);
    if (lane == 0) add_contact(a, q, a0, a1, a2);
}

template <class R>
__global__ void k_fc11(StepArgs<R> a, int64_t first, int64_t n, int64_t nbrows, const int32_t *nb11,
                       const int32_t *roff, const int32_t *rev, const double *dens, CLawF law, const int32_t *act,
                       int64_t nact) {
    const int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= nact) return;
    const int64_t li = act ? act[t] : t;
    const int64_t p = first + li;
    const int32_t o = roff[li], e = roff[li + 1];
    if (o == e && nb11[li] < 0) return;
    double yp0, yp1, yp2, a0 = 0, a1 = 0, a2 = 0, F0, F1, F2;
    ypos(a, p, yp0, yp1, yp2);
    const double den = dens[p], vol = a.x64[p].w;
    for (int32_t r = o + lane; r < e; r += 32) {
        double yi0, yi1, yi2;
        ypos(a, rev[r], yi0, yi1, yi2);
        cfn(law, yi0 - yp0, yi1 - yp1, yi2 - yp2, F0, F1, F2);
        a0 -= F0 * (vol / den);
        a1 -= F1 * (vol / den);
        a2 -= F2 * (vol / den);
    }
    for (int64_t k0 = 0; k0 < nbrows; k0 += 32) {
        const int64_t k = k0 + lane;
        const int32_t q = k < nbrows ? nb11[k * n + li] : -1;
        const uint32_t stop = __ballot_sync(0xffffffffu, q < 0);
        const int nlive = stop ? __ffs(stop) - 1 : 32;
        if (lane < nlive) {
            double yq0, yq1, yq2;
            ypos(a, q, yq0, yq1, yq2);
            cfn(law, yp0 - yq0, yp1 - yq1, yp2 - yq2, F0, F1, F2);
            const double s = a.x64[q].w / den;
            a0 += F0 * s;
            a1 += F1 * s;
            a2 += F2 * s;
        }
        if (stop) break;
    }
    warp_sum3(a0, a1, a2);
    if (lane == 0) add_contact(a, p, a0, a1, a2);
}

// ----------------------------------------------------------------------
// host-side state
// ----------------------------------------------------------------------
template <class R>
struct Fast {
    using V4 = typename Tr<R>::V4;
    using V2 = typename Tr<R>::V2;
    DBuf<V4> xu[2], v, f, p;  // xu: interleaved (x, u) records, 2N entries each
    DBuf<double> ax, ay, az;
    DBuf<R> irho, mass;
    DBuf<V2> mab;
    DBuf<FBlock<R>> fb;
    DBuf<FPair<R>> fp;
    DBuf<uint8_t> bcbits;
    DBuf<int32_t> bcrank;            // per BC, dense over its index range
    std::vector<int64_t> bcrank_off, bcrank_lo;
    DBuf<double> gpart;
    DBuf<GateItem> gitems;
    std::vector<GateItem> gitems_h;
    DBuf<V4> tune;        // autotuner output scratch
    DBuf<double> tune_d;
    DBuf<int32_t> ones;   // all blocks "deformed" while tuning
    DBuf<GridBar> gbar;   // persistent-chunk barrier state
    DBuf<int32_t> serr;   // staged kernels: a staging copy timed out
    DBuf<R> rtd;          // elasto-plastic: 1/sqrt(td_norm2) per particle
    DBuf<V4> cacc;        // contact accelerations of the current step (zero between steps)
    DBuf<int32_t> partner;  // elasto-plastic: reverse-bond slot per slot
    bool persisted = false;
    int cur = 0;
    int wps = 0;          // warps per 32-particle slice (autotuned)
    // CUDA graphs of kGraphSteps velocity-Verlet steps, keyed by the first
    // step's arguments (buffer parity, BC directions) and the gate list.
    struct Graph {
        StepArgs<R> a0;
        std::vector<GateItem> gate;
        int64_t cepoch;  // contact-list generation the captured contact kernels use
        int wps;
        int64_t kernels;  // kernel nodes per replay
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;
    // pinned copy of the device gate flags, read back without stalling
    int32_t *flags_h = nullptr;
    cudaEvent_t flags_ev = nullptr;
    bool flags_pending = false;
    int64_t gate_runs = 0;          // gate steps enqueued since the gate list last changed
    ~Fast() {
        for (auto &g : graphs) cudaGraphExecDestroy(g.exec);
        if (flags_h) cudaFreeHost(flags_h);
        if (flags_ev) cudaEventDestroy(flags_ev);
    }
};
constexpr int kGraphSteps = 32;
static_assert(kGraphSteps % 2 == 0, "a replay must keep the record-buffer parity");

// Kernel shape, chosen by the autotuner: cfg = 10 * WPS + U (warps per
// slice, bonds in flight per thread).  FP32 tries U in {2, 4}, FP64 {1, 2}.
template <class R>
struct Unroll {
    static constexpr int LO = sizeof(R) == 4 ? 2 : 1;
    static constexpr int HI = sizeof(R) == 4 ? 4 : 2;
};

// Launch of a bond kernel with programmatic stream serialization (the
// kernel enters through pdl_enter); PD_NO_PDL=1 gives ordinary launches.
template <class... P>
inline void launch_dep(void (*kern)(P...), unsigned grid, unsigned block, cudaStream_t st, P... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    const char *off = std::getenv("PD_NO_PDL");
    cfg.attrs = at;
    cfg.numAttrs = (off && std::strcmp(off, "1") == 0) ? 0 : 1;
    cudaLaunchKernelEx(&cfg, kern, args...);
}

template <class R, int MODE, int U, bool EPK = false>
void launch_step_u(cudaStream_t st, int wps, const StepArgs<R> &a) {
    const int64_t slices = (a.N + 31) / 32;
    const unsigned g1 = (unsigned)(a.swz_g ? (int64_t)a.swz_g * a.swz_k : slices);  // one slice per block
    switch (wps) {
        case 1: launch_dep(k_step<R, 1, U, MODE, EPK>, (unsigned)((slices + 3) / 4), 128, st, a); break;
        case 2: launch_dep(k_step<R, 2, U, MODE, EPK>, (unsigned)((slices + 1) / 2), 128, st, a); break;
        case 4: launch_dep(k_step<R, 4, U, MODE, EPK>, g1, 128, st, a); break;
        default: launch_dep(k_step<R, 8, U, MODE, EPK>, g1, 256, st, a); break;
    }
    note_launch();
}

// Elasto-plastic td_norm2 pass (one unroll: U = LO).
template <class R>
void launch_td(cudaStream_t st, int cfg, const StepArgs<R> &a) {
    constexpr int U = Unroll<R>::LO;
    const int64_t slices = (a.N + 31) / 32;
    const unsigned g1 = (unsigned)(a.swz_g ? (int64_t)a.swz_g * a.swz_k : slices);
    switch (cfg % 100 / 10) {
        case 1: launch_dep(k_td<R, 1, U>, (unsigned)((slices + 3) / 4), 128, st, a); break;
        case 2: launch_dep(k_td<R, 2, U>, (unsigned)((slices + 1) / 2), 128, st, a); break;
        case 4: launch_dep(k_td<R, 4, U>, g1, 128, st, a); break;
        default: launch_dep(k_td<R, 8, U>, g1, 256, st, a); break;
    }
    note_launch();
}

// Staged shapes (cfg >= 100, FP32C): one block of WPS warps per slice,
// a.stage_bytes of dynamic shared memory.
template <int MODE>
void launch_step_st(cudaStream_t st, int cfg, StepArgs<float> a) {
    a.swz_g = 0;  // block b stages and walks slice b
    const unsigned slices = (unsigned)((a.N + 31) / 32);
    const size_t sm = (size_t)a.stage_bytes;
    switch (cfg % 100) {
        case 42: k_step_st<4, 2, MODE><<<slices, 128, sm, st>>>(a); break;
        case 44: k_step_st<4, 4, MODE><<<slices, 128, sm, st>>>(a); break;
        case 82: k_step_st<8, 2, MODE><<<slices, 256, sm, st>>>(a); break;
        default: k_step_st<8, 4, MODE><<<slices, 256, sm, st>>>(a); break;
    }
    note_launch();
}

inline void launch_theta_st(cudaStream_t st, int cfg, StepArgs<float> a) {
    a.swz_g = 0;  // block b stages and walks slice b
    const unsigned slices = (unsigned)((a.N + 31) / 32);
    const size_t sm = (size_t)a.stage_bytes;
    switch (cfg % 100) {
        case 42: k_theta_st<4, 2><<<slices, 128, sm, st>>>(a); break;
        case 44: k_theta_st<4, 4><<<slices, 128, sm, st>>>(a); break;
        case 82: k_theta_st<8, 2><<<slices, 256, sm, st>>>(a); break;
        default: k_theta_st<8, 4><<<slices, 256, sm, st>>>(a); break;
    }
    note_launch();
}

// The staged kernels may use up to kStageMaxRecords records of dynamic
// shared memory; raise their limit once per device (the attribute is a
// per-device setting), with `device` current.
constexpr int kAttrDevices = 64;
std::mutex g_attr_mutex;
bool g_attr_done[kAttrDevices] = {};
cudaError_t g_attr_status[kAttrDevices] = {};
inline cudaError_t staged_kernel_attrs(int device) {
    if (device < 0 || device >= kAttrDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    if (g_attr_done[device]) return g_attr_status[device];
    cudaError_t status = [] {
        const int bytes = (int)(kStageMaxRecords * 32);
        cudaError_t e = cudaSuccess;
        auto set = [&](const void *k) {
            const cudaError_t r = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            if (r != cudaSuccess && e == cudaSuccess) e = r;
        };
#define PD_STAGED_ATTRS(W, U)                                                                               \
    set((const void *)k_step_st<W, U, 0>);                                                                  \
    set((const void *)k_step_st<W, U, 1>);                                                                  \
    set((const void *)k_step_st<W, U, 2>);                                                                  \
    set((const void *)k_theta_st<W, U>);
        PD_STAGED_ATTRS(4, 2)
        PD_STAGED_ATTRS(4, 4)
        PD_STAGED_ATTRS(8, 2)
        PD_STAGED_ATTRS(8, 4)
#undef PD_STAGED_ATTRS
        return e;
    }();
    g_attr_done[device] = true;
    g_attr_status[device] = status;
    return status;
}

template <class R, int MODE>
void launch_step(cudaStream_t st, int cfg, const StepArgs<R> &a) {
    if (a.ep) {  // elasto-plastic kernels: one unroll, no staging
        launch_step_u<R, MODE, Unroll<R>::LO, true>(st, cfg % 100 / 10, a);
        return;
    }
    if constexpr (sizeof(R) == 4) {
        if (cfg >= 100) {
            launch_step_st<MODE>(st, cfg, a);
            return;
        }
    }
    if (cfg % 10 == Unroll<R>::LO) launch_step_u<R, MODE, Unroll<R>::LO>(st, cfg / 10, a);
    else launch_step_u<R, MODE, Unroll<R>::HI>(st, cfg / 10, a);
}

template <class R, int U>
void launch_theta_u(cudaStream_t st, int wps, const StepArgs<R> &a) {
    const int64_t slices = (a.N + 31) / 32;
    const unsigned g1 = (unsigned)(a.swz_g ? (int64_t)a.swz_g * a.swz_k : slices);  // one slice per block
    switch (wps) {
        case 1: launch_dep(k_theta<R, 1, U>, (unsigned)((slices + 3) / 4), 128, st, a); break;
        case 2: launch_dep(k_theta<R, 2, U>, (unsigned)((slices + 1) / 2), 128, st, a); break;
        case 4: launch_dep(k_theta<R, 4, U>, g1, 128, st, a); break;
        default: launch_dep(k_theta<R, 8, U>, g1, 256, st, a); break;
    }
    note_launch();
}

template <class R>
void launch_theta(cudaStream_t st, int cfg, const StepArgs<R> &a) {
    if constexpr (sizeof(R) == 4) {
        if (cfg >= 100) {
            launch_theta_st(st, cfg, a);
            return;
        }
    }
    if (cfg % 10 == Unroll<R>::LO) launch_theta_u<R, Unroll<R>::LO>(st, cfg / 10, a);
    else launch_theta_u<R, Unroll<R>::HI>(st, cfg / 10, a);
}

struct FastHolder {
    int prec = 0;
    Fast<float> f32;
    Fast<double> f64;
    bool dirty = false;  // fast state newer than the FP64 arrays
};

FastHolder *holder(pd_env *env) { return (FastHolder *)env->fast; }

template <class R>
StepArgs<R> args(pd_env *env, Fast<R> &F) {
    StepArgs<R> a;
    std::memset(&a, 0, sizeof(a));  // byte-comparable (graph cache keys)
    a.N = env->N;
    a.xu = F.xu[F.cur].p;
    a.xn = F.xu[1 - F.cur].p;
    a.ax = F.ax.p;
    a.ay = F.ay.p;
    a.az = F.az.p;
    a.v = F.v.p;
    a.f = F.f.p;
    a.p = F.p.p;
    a.irho = F.irho.p;
    a.mass = F.mass.p;
    a.mab = F.mab.p;
    a.tinfo = env->tinfo.p;
    a.cnt = env->cnt.p;
    a.nbr = env->nbr.p;
    a.si = env->sinfo.p;
    a.splan_off = env->splan_off.p;
    a.splan = env->splan.p;
    a.spos = env->spos.p;
    a.serr = F.serr.p;
    a.stage_bytes = (int32_t)(env->splan_max * 32);
    a.ep = 0;
    for (const auto &b : env->hb)
        if (b.kind == PD_MAT_ELASTO_PLASTIC) a.ep = 1;
    if (a.ep) {
        a.edp_in = env->edp[env->ecur].p;
        a.edp_out = env->edp[1 - env->ecur].p;
        a.rtd = F.rtd.p;
        a.partner = F.partner.p;
    }
    const char *sw = std::getenv("PD_SWIZZLE");
    if (!(sw && std::strcmp(sw, "0") == 0)) {  // on unless PD_SWIZZLE=0
        if (env->sm_count == 0) cudaDeviceGetAttribute(&env->sm_count, cudaDevAttrMultiProcessorCount, env->device);
        const int sms = env->sm_count;
        const int64_t S = (env->N + 31) / 32;
        if (sms > 0 && S > sms) {
            a.swz_g = sms;
            a.swz_k = (int32_t)((S + sms - 1) / sms);
        }
    }
    a.words = env->words[env->cur].p;
    a.fb = F.fb.p;
    a.fp = F.fp.p;
    a.deformed = env->deformed.p;
    a.all_def = 1;
    for (size_t b = 0; b < env->hb.size(); ++b)
        if (env->hb[b].kind != PD_MAT_SKIP && !env->deformed_h[b]) a.all_def = 0;
    a.x64 = env->x4.p;
    a.bcbits = F.bcbits.p;
    a.c = (R)(env->dt / 2);
    a.dt = env->dt;
    a.nbc = (int)env->hbc.size();
    for (size_t k = 0; k < env->hbc.size() && k < (size_t)kMaxFastBC; ++k) {
        const HostBC &h = env->hbc[k];
        FBC &b = a.bc[k];
        b.kind = h.kind;
        b.dims = h.dims;
        for (int d = 0; d < 3; ++d) {
            b.rate[d] = h.rate[d];
            b.scale[d] = h.scale[d];
            b.fix[d] = h.fix[d];
            b.lo[d] = h.lo[d];
            b.hi[d] = h.hi[d];
        }
        b.has_limits = h.has_limits;
        b.n = env->bcs[k].n;
        b.idx = env->bcs[k].idx.p;
        b.last = env->bcs[k].last.p;
        b.sn = env->bcs[k].sn;
        b.sidx = env->bcs[k].sidx.p;
        b.rank_lo = k < F.bcrank_lo.size() ? F.bcrank_lo[k] : 0;
        b.rank = F.bcrank.p ? F.bcrank.p + (k < F.bcrank_off.size() ? F.bcrank_off[k] : 0) : nullptr;
    }
    a.ts = env->ts;
    return a;
}

uint32_t dir_bits(const pd_env *env) {
    uint32_t m = 0;
    for (size_t k = 0; k < env->hbc.size(); ++k)
        if (env->hbc[k].dir < 0) m |= 1u << k;
    return m;
}

template <class R>
pd_status init_fast(pd_env *env, Fast<R> &F) {
    const int64_t N = env->N;
    if (!F.xu[0].p) {
        if (sizeof(R) == 4) {
            PD_TRY(F.ax.alloc(N));
            PD_TRY(F.ay.alloc(N));
            PD_TRY(F.az.alloc(N));
        }
        PD_TRY(F.xu[0].alloc(2 * N));
        PD_TRY(F.xu[1].alloc(2 * N));
        PD_TRY(F.v.alloc(N));
        PD_TRY(F.f.alloc(N));
        PD_TRY(F.p.alloc(N));
        PD_TRY(F.irho.alloc(N));
        PD_TRY(F.mass.alloc(N));
        PD_TRY(F.mab.alloc(N));
        PD_TRY(F.bcbits.alloc(N));
        if (!env->hc.empty()) {
            PD_TRY(F.cacc.alloc(N));
            CK(cudaMemsetAsync(F.cacc.p, 0, N * sizeof(typename Tr<R>::V4), env->st));
        }
        // parameters in the working precision
        std::vector<FBlock<R>> fb;
        std::vector<FPair<R>> fp;
        for (const auto &b : env->hb) {
            FBlock<R> d{};
            d.kind = b.kind;
            d.nt = b.nt;
            d.pair_base = (int32_t)fp.size();
            d.c11 = (R)b.c[0];
            fb.push_back(d);
            for (int j = 0; j < b.nt; ++j)
                for (int i = 0; i < b.nt; ++i) {
                    size_t e = (size_t)i + (size_t)j * b.nt;
                    FPair<R> pp{};
                    pp.cs = (R)b.cs[e];
                    const bool ep = b.kind == PD_MAT_ELASTO_PLASTIC;
                    pp.k35 = (R)(ep ? 3 * b.K[e] : 3 * b.K[e] - 5 * b.G[e]);
                    pp.g15 = (R)(15 * b.G[e]);
                    pp.psi = ep ? (R)std::sqrt(2 * b.psi[e]) : R(0);
                    fp.push_back(pp);
                }
        }
        PD_TRY(F.fb.alloc(fb.size()));
        PD_TRY(F.fp.alloc(fp.size()));
        if (!F.serr.p) {
            PD_TRY(F.serr.alloc(1));
            CK(cudaMemsetAsync(F.serr.p, 0, sizeof(int32_t), env->st));
        }
        CK(cudaMemcpyAsync(F.fb.p, fb.data(), fb.size() * sizeof(FBlock<R>), cudaMemcpyHostToDevice, env->st));
        CK(cudaMemcpyAsync(F.fp.p, fp.data(), fp.size() * sizeof(FPair<R>), cudaMemcpyHostToDevice, env->st));
        std::vector<uint8_t> bits(N, 0);
        for (size_t k = 0; k < env->hbc.size(); ++k)
            for (int64_t e : env->hbc[k].env_idx) bits[env->map_h[e]] |= (uint8_t)(1u << k);
        CK(cudaMemcpyAsync(F.bcbits.p, bits.data(), N, cudaMemcpyHostToDevice, env->st));
        // rank tables: BC k's particle p sits at rank[k][p - lo[k]] of its
        // ascending index list (no search in the step kernel)
        std::vector<int32_t> rank;
        F.bcrank_off.clear();
        F.bcrank_lo.clear();
        for (size_t k = 0; k < env->hbc.size(); ++k) {
            const auto &ei = env->hbc[k].env_idx;
            F.bcrank_off.push_back((int64_t)rank.size());
            if (ei.empty()) {
                F.bcrank_lo.push_back(0);
                continue;
            }
            const int64_t lo = env->map_h[ei.front()], hi = env->map_h[ei.back()];
            F.bcrank_lo.push_back(lo);
            const size_t base = rank.size();
            rank.resize(base + (size_t)(hi - lo + 1), -1);
            for (size_t r = 0; r < ei.size(); ++r) rank[base + (size_t)(env->map_h[ei[r]] - lo)] = (int32_t)r;
        }
        PD_TRY(F.bcrank.alloc(std::max<size_t>(rank.size(), 1)));
        if (!rank.empty())
            CK(cudaMemcpyAsync(F.bcrank.p, rank.data(), rank.size() * 4, cudaMemcpyHostToDevice, env->st));
        CK(cudaStreamSynchronize(env->st));
    }
    F.cur = 0;
    StepArgs<R> ai = args(env, F);  // FP64 reads x4 in place; FP32C fills F.x
    k_import<R><<<gridn(env->N, 256), 256, 0, env->st>>>(env->N, env->x4.p, env->y.p, env->v.p, env->f.p, env->p.p,
                                                         env->mass.p, env->dens.p, env->mth.p, env->tinfo.p,
                                                         env->blocks_d.p, ai);
    note_launch();
    CK(cudaGetLastError());
    if (ai.ep) {
        PD_TRY(F.rtd.alloc(env->N));
        PD_TRY(F.partner.alloc(std::max<int64_t>(env->nnz, 1)));
        k_partner<R><<<gridn(env->N), kT, 0, env->st>>>(ai, env->fam.p, F.partner.p);
        note_launch();
        CK(cudaGetLastError());
    }
    return PD_OK;
}

template <class R>
pd_status gate_prepare(pd_env *env, Fast<R> &F) {
    std::vector<GateItem> items;
    for (size_t b = 0; b < env->hb.size() && !env->gate_hold; ++b) {
        const HostBlock &hb = env->hb[b];
        if (hb.kind == PD_MAT_SKIP || env->deformed_h[b]) continue;
        items.push_back(GateItem{hb.first_int, hb.n, (int32_t)b, 0});
    }
    if (F.gitems_h.size() != items.size() ||
        std::memcmp(F.gitems_h.data(), items.data(), items.size() * sizeof(GateItem)) != 0) {
        if (!items.empty()) {
            const int ni = (int)items.size();
            const int gx = std::max(1, std::min(kGB, (kGB * 8) / ni));
            PD_TRY(grow(F.gitems, (int64_t)items.size()));
            PD_TRY(grow(F.gpart, 3 * (int64_t)ni * gx));
            CK(cudaMemcpyAsync(F.gitems.p, items.data(), items.size() * sizeof(GateItem), cudaMemcpyHostToDevice,
                               env->st));
            CK(cudaStreamSynchronize(env->st));
        }
        F.gitems_h = items;
        F.gate_runs = 0;
    }
    return PD_OK;
}

// Deformed gate of the blocks in F.gitems_h (prepared by gate_prepare):
// kernel launches only, so it can be captured in a graph.
template <class R>
void gate_launch(pd_env *env, StepArgs<R> &a, Fast<R> &F) {
    if (F.gitems_h.empty()) return;
    const int ni = (int)F.gitems_h.size();
    const int gx = std::max(1, std::min(kGB, (kGB * 8) / ni));
    k_fgate_partial<R><<<dim3(gx, ni), kGT, 0, env->st>>>(a, F.gitems.p, gx, F.gpart.p);
    k_fgate_final<<<(ni + 127) / 128, 128, 0, env->st>>>(F.gitems.p, ni, gx, F.gpart.p, env->deformed.p);
    note_launch();
    note_launch();
}

template <class R>
pd_status gate_if_needed(pd_env *env, StepArgs<R> &a, Fast<R> &F) {
    PD_TRY(gate_prepare(env, F));
    gate_launch(env, a, F);
    if (!F.gitems_h.empty()) ++F.gate_runs;
    return PD_OK;
}

// Refresh of the host copy of the gate flags: issue an async read-back
// once a gate step has been enqueued, and take its result on a later call.
// Without wait the result is taken only once it has landed.  With wait
// (a blocking stepping call) the pending read is waited for: the host otherwise runs so far ahead of the device that a whole
// call's replays are enqueued before the read lands, each still carrying
// the gate kernels after the block has deformed.  The wait leaves the
// replay enqueued after the read in flight, so the device does not idle.
template <class R>
pd_status poll_gate_flags(pd_env *env, Fast<R> &F, bool wait) {
    if (F.gitems_h.empty()) return PD_OK;
    const size_t nb = env->hb.size();
    if (!F.flags_h) {
        CK(cudaMallocHost(&F.flags_h, nb * sizeof(int32_t)));
        CK(cudaEventCreateWithFlags(&F.flags_ev, cudaEventDisableTiming));
    }
    if (F.flags_pending) {
        const cudaError_t q =
            wait ? cudaEventSynchronize(F.flags_ev) : cudaEventQuery(F.flags_ev);
        if (q == cudaErrorNotReady) return PD_OK;
        if (q != cudaSuccess) return cuda_fail(q, "gate flag read-back", __FILE__, __LINE__);
        F.flags_pending = false;
        // drop the gate once every listed block has deformed (a partial
        // change would only cost a re-capture; the kernels skip deformed
        // blocks by themselves)
        for (const GateItem &it : F.gitems_h)
            if (!F.flags_h[it.block]) return PD_OK;
        for (size_t b = 0; b < nb; ++b)
            if (F.flags_h[b]) env->deformed_h[b] = 1;
        return gate_prepare(env, F);
    }
    if (F.gate_runs == 0) return PD_OK;  // no gate step since the list was set: nothing new to read
    CK(cudaMemcpyAsync(F.flags_h, env->deformed.p, nb * sizeof(int32_t), cudaMemcpyDeviceToHost, env->st));
    CK(cudaEventRecord(F.flags_ev, env->st));
    F.flags_pending = true;
    return PD_OK;
}

template <class R>
pd_status contacts_fast(pd_env *env, StepArgs<R> &a) {
    for (size_t k = 0; k < env->hc.size(); ++k) {
        const HostContact &hc = env->hc[k];
        DevContact &dc = env->contacts[k];
        if (!dc.has_neighs) continue;
        CLawF law{hc.equi_dist, hc.exponent, hc.stiffness};
        const bool lists = dc.nact1 >= 0;
        const int64_t n1 = lists ? dc.nact1 : dc.n1;
        const int32_t *a1 = lists ? dc.act1.p : nullptr;
        if (hc.kind == PD_CONTACT_12) {
            const int64_t n2 = lists ? dc.nact2 : dc.n2;
            const int32_t *a2 = lists ? dc.act2.p : nullptr;
            if (n1 > 0) {
                k_fc12_1<R><<<gridn(32 * n1, 256), 256, 0, env->st>>>(a, dc.first1, dc.n1, dc.rows, dc.nb.p,
                                                                      env->dens.p, law, a1, n1);
                note_launch();
            }
            if (n2 > 0) {
                k_fc12_2<R><<<gridn(32 * n2, 256), 256, 0, env->st>>>(a, dc.first2, dc.n2, dc.rev_off.p,
                                                                      dc.rev.p, env->dens.p, law, a2, n2);
                note_launch();
            }
        } else if (n1 > 0) {
            k_fc11<R><<<gridn(32 * n1, 256), 256, 0, env->st>>>(a, dc.first1, dc.n1, dc.nbrows, dc.nb.p,
                                                                dc.rev_off.p, dc.rev.p, env->dens.p, law, a1, n1);
            note_launch();
        }
    }
    CK(cudaGetLastError());
    return PD_OK;
}

template <class V4>
__global__ void k_czero(V4 *cacc, int64_t first, const int32_t *act, int64_t n) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    cacc[first + (act ? act[t] : t)] = V4{};
}

// Clears the entries the contact kernels wrote (their particle lists), so
// the contact acceleration array is zero between steps.
template <class V4>
void contacts_clear(pd_env *env, V4 *cacc) {
    for (size_t k = 0; k < env->hc.size(); ++k) {
        const DevContact &dc = env->contacts[k];
        if (!dc.has_neighs) continue;
        const bool lists = dc.nact1 >= 0;
        const int64_t n1 = lists ? dc.nact1 : dc.n1;
        if (n1 > 0) {
            k_czero<V4><<<gridn(n1, 256), 256, 0, env->st>>>(cacc, dc.first1, lists ? dc.act1.p : nullptr, n1);
            note_launch();
        }
        if (env->hc[k].kind == PD_CONTACT_12) {
            const int64_t n2 = lists ? dc.nact2 : dc.n2;
            if (n2 > 0) {
                k_czero<V4><<<gridn(n2, 256), 256, 0, env->st>>>(cacc, dc.first2, lists ? dc.act2.p : nullptr, n2);
                note_launch();
            }
        }
    }
}

bool any_lps(const pd_env *env) {
    for (const auto &b : env->hb)
        if (b.kind == PD_MAT_ORDINARY_STATE_BASED) return true;
    return false;
}

bool any_ep(const pd_env *env) {
    for (const auto &b : env->hb)
        if (b.kind == PD_MAT_ELASTO_PLASTIC) return true;
    return false;
}

// The dilatation pass runs for state-based and elasto-plastic blocks.
bool need_theta(const pd_env *env) { return any_lps(env) || any_ep(env); }

// One force evaluation: dilatation, the elasto-plastic td_norm2 pass, and
// the step kernel; then the plastic strain buffers swap.
template <class R, int MODE>
void launch_force(pd_env *env, cudaStream_t st, int cfg, const StepArgs<R> &a, bool theta) {
    if (theta) launch_theta(st, cfg, a);
    if (a.ep) launch_td(st, cfg, a);
    launch_step<R, MODE>(st, cfg, a);
    if (a.ep) env->ecur = 1 - env->ecur;
}

// Project autotuner: times every kernel shape on the environment itself
// (captured graphs of full steps on scratch copies of the state they
// write) and keeps the fastest.  Results are cached for the life of the
// process per device and problem class: particle count in steps of
// 2^(1/2) (~41 %), bond slots per particle in steps of 8, precision and
// staging mode, and the passes present (dilatation, td_norm2), so
// environments of similar sizes built one after another on a device tune
// once per class.  (Served jobs do not come here: the server fixes their
// shapes from their sizes.)
std::mutex g_tune_mutex;
std::map<std::tuple<int, int64_t, int64_t, int, int>, int> g_tune_cache;

template <class R>
pd_status autotune(pd_env *env, Fast<R> &F) {
    if (F.wps) return PD_OK;
    // staged shapes: FP32C, 4 or 8 warps per slice, when some slice has a plan
    const bool ep = any_ep(env);
    const bool can_stage = sizeof(R) == 4 && env->splan_slices > 0 && !ep;
    if (can_stage) CK(staged_kernel_attrs(env->device));
    auto staged_ok = [&](int w) { return can_stage && (w == 4 || w == 8); };
    if (env->shape) {  // pd_env_set_kernel_shape (+ pd_env_set_record_staging)
        F.wps = env->shape + (env->staging == 1 && staged_ok(env->shape / 10) ? 100 : 0);
        return PD_OK;
    }
    const bool lps = need_theta(env);
    const int64_t size_class = (int64_t)std::floor(2.0 * std::log2((double)std::max<int64_t>(env->N, 1)));
    const int64_t slot_class = env->nnz / std::max<int64_t>(env->N, 1) / 8;
    const auto key = std::make_tuple(env->device, size_class, slot_class, env->precision * 4 + env->staging + 1,
                                     (int)lps + 2 * (int)ep);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            F.wps = it->second;
            return PD_OK;
        }
    }
    if (const char *fixed = std::getenv("PD_KERNEL_SHAPE")) {  // "WPS,U[,staged]" overrides the tuner
        int w = 0, u = 0, sg = 0;
        const int n = std::sscanf(fixed, "%d,%d,%d", &w, &u, &sg);
        if (n >= 2 && (w == 1 || w == 2 || w == 4 || w == 8) && (u == Unroll<R>::LO || u == Unroll<R>::HI)) {
            F.wps = 10 * w + u + (n == 3 && sg == 1 && staged_ok(w) ? 100 : 0);
            return PD_OK;
        }
    }
    // The timed kernels are the full step (dilatation; force, integration,
    // BCs and bond breaking, MODE 1) writing every output -- velocities,
    // records, bond words, BC positions -- into scratch copies, so the
    // environment's state is left untouched.
    const int64_t N = env->N;
    PD_TRY(F.tune.alloc(5 * N));
    PD_TRY(F.tune_d.alloc(3 * N));
    CK(cudaMemsetAsync(F.tune.p, 0, 5 * N * sizeof(typename Tr<R>::V4), env->st));
    CK(cudaMemsetAsync(F.tune_d.p, 0, 3 * N * sizeof(double), env->st));
    std::vector<int32_t> ones(env->hb.size(), 1);
    PD_TRY(F.ones.alloc(ones.size()));
    CK(cudaMemcpyAsync(F.ones.p, ones.data(), ones.size() * 4, cudaMemcpyHostToDevice, env->st));
    StepArgs<R> a = args(env, F);
    a.v = F.tune.p;
    a.f = F.tune.p + N;
    a.p = F.tune.p + 2 * N;
    a.xn = F.tune.p + 3 * N;
    a.ax = F.tune_d.p;
    a.ay = F.tune_d.p + N;
    a.az = F.tune_d.p + 2 * N;
    a.deformed = F.ones.p;
    a.all_def = 1;
    const int64_t nwords = std::max<int64_t>(env->nnz / 32, 1);
    DBuf<uint32_t> twords;
    PD_TRY(twords.alloc(nwords));
    CK(cudaMemcpyAsync(twords.p, a.words, nwords * 4, cudaMemcpyDeviceToDevice, env->st));
    a.words = twords.p;
    DBuf<double> tedp;
    DBuf<R> trtd;
    if (a.ep) {  // plastic strain and td_norm2 of the timed steps go to scratch
        PD_TRY(tedp.alloc(std::max<int64_t>(env->nnz, 1)));
        PD_TRY(trtd.alloc(N));
        a.edp_out = tedp.p;
        a.rtd = trtd.p;
    }
    int64_t nlast = 0;
    for (int k = 0; k < a.nbc; ++k)
        if (a.bc[k].last) nlast += a.bc[k].n;
    DBuf<double4> tlast;
    PD_TRY(tlast.alloc(std::max<int64_t>(nlast, 1)));
    for (int k = 0, off = 0; k < a.nbc; ++k) {
        if (!a.bc[k].last) continue;
        CK(cudaMemcpyAsync(tlast.p + off, a.bc[k].last, a.bc[k].n * sizeof(double4), cudaMemcpyDeviceToDevice,
                           env->st));
        a.bc[k].last = tlast.p + off;
        off += (int)a.bc[k].n;
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best = 1e30f;
    int best_w = 40 + Unroll<R>::LO;
    std::vector<int> shapes;
    for (int wps : {1, 2, 4, 8})
        for (int u : {Unroll<R>::LO, Unroll<R>::HI}) {
            if (ep && u != Unroll<R>::LO) continue;  // the elasto-plastic kernels have one unroll
            if (env->staging != 1 || !staged_ok(wps)) shapes.push_back(10 * wps + u);
            if (env->staging >= 1 && staged_ok(wps)) shapes.push_back(100 + 10 * wps + u);
        }
    // Each shape runs as the stepping loop does: a captured graph of
    // kTuneSteps steps (fewer for large problems, whose steps are long
    // enough to time), replayed once to warm up and then timed in two
    // sweeps over the shapes, best of the two per shape.
    const int kTuneSteps = N > 200000 ? 3 : N > 50000 ? 6 : 12;
    std::vector<cudaGraphExec_t> ex(shapes.size(), nullptr);
    auto release = [&] {
        for (auto &g : ex)
            if (g) cudaGraphExecDestroy(g);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    };
    for (size_t i = 0; i < shapes.size(); ++i) {
        cudaGraph_t graph = nullptr;
        cudaError_t err = cudaStreamBeginCapture(env->st, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) {
            for (int r = 0; r < kTuneSteps; ++r) {
                if (lps) launch_theta(env->st, shapes[i], a);
                if (a.ep) launch_td(env->st, shapes[i], a);
                launch_step<R, 1>(env->st, shapes[i], a);
            }
            err = cudaStreamEndCapture(env->st, &graph);
        }
        if (err == cudaSuccess) err = cudaGraphInstantiate(&ex[i], graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (err == cudaSuccess) err = cudaGraphLaunch(ex[i], env->st);
        if (err != cudaSuccess) {
            release();
            return cuda_fail(err, "autotune", __FILE__, __LINE__);
        }
    }
    std::vector<float> t(shapes.size(), 1e30f);
    for (int sweep = 0; sweep < 2; ++sweep)
        for (size_t i = 0; i < shapes.size(); ++i) {
            cudaEventRecord(e0, env->st);
            cudaGraphLaunch(ex[i], env->st);
            cudaEventRecord(e1, env->st);
            cudaError_t err = cudaEventSynchronize(e1);
            if (err != cudaSuccess) {
                release();
                return cuda_fail(err, "autotune", __FILE__, __LINE__);
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            t[i] = std::min(t[i], ms);
        }
    for (size_t i = 0; i < shapes.size(); ++i)
        if (t[i] < best) {
            best = t[i];
            best_w = shapes[i];
        }
    if (std::getenv("PD_TUNE_LOG")) {
        std::fprintf(stderr, "pd autotune N=%lld:", (long long)env->N);
        for (size_t i = 0; i < shapes.size(); ++i)
            std::fprintf(stderr, " %s%d,%d=%.2fus", shapes[i] >= 100 ? "s" : "", shapes[i] % 100 / 10, shapes[i] % 10,
                         1e3f * t[i] / kTuneSteps);
        std::fprintf(stderr, " -> %d\n", best_w);
    }
    release();
    CK(cudaGetLastError());
    F.tune.reset();
    F.tune_d.reset();
    F.wps = best_w;
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = best_w;
    return PD_OK;
}

// ScaleFixWaitBC.jl:63-68 check! on the throughput state: scale the
// scalebool particles' positions about the fix point (through their FP64
// displacement), then re-read BC.last from the positions.
template <class R>
__global__ void k_fscale(StepArgs<R> a, int k) {
    const FBC &b = a.bc[k];
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= b.sn) return;
    const int64_t p = b.sidx[j];
    double u[3];
    load_u(a, p, u[0], u[1], u[2]);
    const double4 x = a.x64[p];
    const double xx[3] = {x.x, x.y, x.z};
    for (int d = 0; d < 3; ++d) {
        if (!((b.dims >> d) & 1)) continue;
        const double g = sqrt(1.0 + (2.0 * b.scale[d]) * a.dt);
        u[d] = ((xx[d] + u[d]) - b.fix[d]) * g + b.fix[d] - xx[d];
    }
    // the current record buffer holds the state between steps
    StepArgs<R> c = a;
    c.xn = const_cast<typename Tr<R>::V4 *>(a.xu);
    store_u(c, p, u[0], u[1], u[2]);
}

template <class R>
__global__ void k_fsnapshot(StepArgs<R> a, int k) {
    const FBC &b = a.bc[k];
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= b.n) return;
    const int64_t p = b.idx[j];
    double u0, u1, u2;
    load_u(a, p, u0, u1, u2);
    const double4 x = a.x64[p];
    double4 last = b.last[j];
    if (b.dims & 1) last.x = x.x + u0;
    if (b.dims & 2) last.y = x.y + u1;
    if (b.dims & 4) last.z = x.z + u2;
    b.last[j] = last;
}

// Any ScaleFixWait check! at this time_step?
bool scale_check_due(const pd_env *env) {
    for (const auto &h : env->hbc)
        if (h.scales_at(env->ts)) return true;
    return false;
}

bool time_dependent_bcs(const pd_env *env) {
    for (const auto &h : env->hbc)
        if (h.kind == PD_BC_DELTA_SCALE || h.kind == PD_BC_SCALE_FIX_WAIT) return true;
    return false;
}

// check!(env) then time_step += 1 (velocity_verlet.jl:81-85): ToFro
// direction flips when time_step > applyafter and time_step % freq == 0.
void advance_bc_clock(pd_env *env) {
    for (auto &h : env->hbc) {
        if (h.kind != PD_BC_TOFRO) continue;
        const double r = std::fmod((double)env->ts, h.freq);
        if ((env->ts > h.applyafter) && (r == 0.0)) h.dir = -h.dir;
    }
    env->ts += 1;
}

// True when none of the next n steps flips a BC direction.
bool flip_free_steps(const pd_env *env, int64_t n) {
    for (const auto &h : env->hbc) {
        if (h.kind != PD_BC_TOFRO) continue;
        for (int64_t k = 0; k < n; ++k) {
            const int64_t ts = env->ts + k;
            if ((ts > h.applyafter) && std::fmod((double)ts, h.freq) == 0.0) return false;
        }
    }
    return true;
}

// Launch kGraphSteps full steps (MODE 1) from the current state: the
// cached graph for these arguments, captured on first use.
template <class R>
pd_status replay_graph(pd_env *env, Fast<R> &F, bool lps) {
    cudaStream_t st = env->st;
    StepArgs<R> a0 = args(env, F);
    a0.dir_vel = a0.dir_pos = dir_bits(env);
    a0.ts = 0;  // graphs run only without time-dependent BCs
    typename Fast<R>::Graph *hit = nullptr;
    for (auto &g : F.graphs)
        if (g.wps == F.wps && g.cepoch == env->contact_epoch && g.gate.size() == F.gitems_h.size() &&
            std::memcmp(&g.a0, &a0, sizeof(a0)) == 0 &&
            std::memcmp(g.gate.data(), F.gitems_h.data(), g.gate.size() * sizeof(GateItem)) == 0) {
            hit = &g;
            break;
        }
    if (!hit) {
        if (F.graphs.size() >= 8) {
            for (auto &g : F.graphs) cudaGraphExecDestroy(g.exec);
            F.graphs.clear();
        }
        const int cur0 = F.cur, ecur0 = env->ecur;
        const int64_t n0 = launch_count();
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < kGraphSteps; ++k) {
            StepArgs<R> a = args(env, F);
            a.dir_vel = a.dir_pos = a0.dir_vel;
            a.ts = 0;
            gate_launch(env, a, F);
            if (env->hc.empty()) {
                launch_force<R, 1>(env, st, F.wps, a, lps);
            } else {
                // as a direct contact step: contact accelerations at this
                // step's positions into F.cacc, the fused step adds them,
                // the touched entries are cleared
                if (lps) launch_theta(st, F.wps, a);
                if (a.ep) launch_td(st, F.wps, a);
                StepArgs<R> b = a;
                b.f = F.cacc.p;
                const pd_status cs = contacts_fast(env, b);
                if (cs != PD_OK) {
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(st, &g);
                    if (g) cudaGraphDestroy(g);
                    F.cur = cur0;
                    env->ecur = ecur0;
                    add_launches(-(launch_count() - n0));
                    return cs;
                }
                a.cacc = F.cacc.p;
                launch_step<R, 1>(st, F.wps, a);
                if (a.ep) env->ecur = 1 - env->ecur;
                contacts_clear(env, F.cacc.p);
            }
            F.cur = 1 - F.cur;
        }
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(st, &graph);
        F.cur = cur0;  // kGraphSteps is even: the parities are unchanged
        env->ecur = ecur0;
        const int64_t kernels = launch_count() - n0;  // captured, not run
        add_launches(-kernels);
        if (ce != cudaSuccess) return cuda_fail(ce, "graph capture", __FILE__, __LINE__);
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) return cuda_fail(ie, "graph instantiate", __FILE__, __LINE__);
        F.graphs.push_back(typename Fast<R>::Graph{a0, F.gitems_h, env->contact_epoch, F.wps, kernels, exec});
        hit = &F.graphs.back();
    }
    CK(cudaGraphLaunch(hit->exec, st));
    add_launches(hit->kernels);
    if (!hit->gate.empty()) F.gate_runs += kGraphSteps;
    for (int k = 0; k < kGraphSteps; ++k) advance_bc_clock(env);
    return PD_OK;
}

// Steps from the current time_step before the next BC direction flip (at most maxn).
int64_t flip_free_run(const pd_env *env, int64_t maxn) {
    int64_t n = 0;
    for (; n < maxn; ++n)
        for (const auto &h : env->hbc)
            if (h.kind == PD_BC_TOFRO && (env->ts + n > h.applyafter) && std::fmod((double)(env->ts + n), h.freq) == 0.0)
                return n;
    return n;
}

// Launch nsteps full steps as one persistent cooperative kernel of at most
// as many blocks as the device holds at once (each block walks several
// slice groups when there are more); *done = false (no block fits) leaves
// the steps to the caller.
template <class R, int WPS, int U, bool LPS>
pd_status persist_try(pd_env *env, Fast<R> &F, int nsteps, bool *done) {
    constexpr int BT = Split<WPS>::BT, SPB = Split<WPS>::SPB;
    void (*kern)(const StepArgs<R>, const StepArgs<R>, int, GridBar *, int64_t) = k_persist<R, WPS, U, LPS>;
    int64_t ngroups = ((env->N + 31) / 32 + SPB - 1) / SPB;
    int per_sm = 0, sms = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BT, 0));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, env->device));
    const int64_t blocks = std::min<int64_t>(ngroups, (int64_t)per_sm * sms);
    if (blocks < 1) {
        *done = false;
        return PD_OK;
    }
    if (!F.gbar.p) {
        PD_TRY(F.gbar.alloc(1));
        CK(cudaMemsetAsync(F.gbar.p, 0, sizeof(GridBar), env->st));
    }
    StepArgs<R> a0 = args(env, F);
    a0.swz_g = 0;  // the cooperative grid covers the slices in order
    a0.dir_vel = a0.dir_pos = dir_bits(env);
    a0.ts = env->ts + 1;
    // even steps read the current record buffer and write the other one
    typename Tr<R>::V4 *b0 = F.xu[F.cur].p, *b1 = F.xu[1 - F.cur].p;
    a0.xu = b0;
    a0.xn = b1;
    StepArgs<R> a1 = a0;
    a1.xu = b1;
    a1.xn = b0;
    GridBar *gb = F.gbar.p;
    void *kargs[] = {&a0, &a1, &nsteps, &gb, &ngroups};
    CK(cudaLaunchCooperativeKernel((const void *)kern, dim3((unsigned)blocks), dim3(BT), kargs, 0, env->st));
    add_launches(1);
    for (int k = 0; k < nsteps; ++k) advance_bc_clock(env);
    if (nsteps & 1) F.cur = 1 - F.cur;
    F.persisted = true;
    *done = true;
    return PD_OK;
}

// The persistent kernel runs the environment's kernel shape (F.wps), so a
// run gives the same numbers whichever launch path each step takes.
template <class R, bool LPS>
pd_status persist_any(pd_env *env, Fast<R> &F, int nsteps, bool *done) {
    constexpr int LO = Unroll<R>::LO, HI = Unroll<R>::HI;
    switch (F.wps % 100) {  // the persistent kernel reads global memory (no staging)
        case 10 + LO: return persist_try<R, 1, LO, LPS>(env, F, nsteps, done);
        case 10 + HI: return persist_try<R, 1, HI, LPS>(env, F, nsteps, done);
        case 20 + LO: return persist_try<R, 2, LO, LPS>(env, F, nsteps, done);
        case 20 + HI: return persist_try<R, 2, HI, LPS>(env, F, nsteps, done);
        case 40 + LO: return persist_try<R, 4, LO, LPS>(env, F, nsteps, done);
        case 40 + HI: return persist_try<R, 4, HI, LPS>(env, F, nsteps, done);
        case 80 + LO: return persist_try<R, 8, LO, LPS>(env, F, nsteps, done);
        default: return persist_try<R, 8, HI, LPS>(env, F, nsteps, done);
    }
}

template <class R>
pd_status vv_chunk(pd_env *env, Fast<R> &F, int64_t nsteps, bool blocking = true) {
    cudaStream_t st = env->st;
    const unsigned grid = gridn(env->N);
    const bool lps = need_theta(env);
    const bool contacts = !env->hc.empty();
    PD_TRY(autotune(env, F));
    const int wps = F.wps;
    {
        StepArgs<R> a = args(env, F);
        a.dir_pos = dir_bits(env);
        k_prologue<R><<<grid, kT, 0, st>>>(a);
        note_launch();
        F.cur = 1 - F.cur;
    }
    // Steps run as replays of a captured graph of kGraphSteps steps while
    // the BC directions stay constant (with contacts: between neighbour
    // updates, which change the contact lists; a graph is keyed by their
    // generation); the rest (direction flips, time-dependent BCs, the last
    // step) launch directly.  With profiling on, timing events bracket each
    // replay (kGraphSteps steps) and the bond kernels of each direct step.
    const bool graphs = !time_dependent_bcs(env) && !std::getenv("PD_NO_GRAPHS");
    // With PD_PERSIST=1, once every block has deformed (no gate), flip-free
    // runs go to one persistent cooperative launch when the grid of the
    // chosen shape fits on the device.  Off by default: on B200 the graph
    // replays measured faster (40 k-particle LPS bar at 2 warps/slice: 44.7
    // against 49.1 us per step; 17.6 k-particle PMB cube: 15.6 against
    // 17.5 us), the grid barriers costing more than graph kernel boundaries.
    const char *pe = std::getenv("PD_PERSIST");
    const bool persist = graphs && !contacts && pe && std::strcmp(pe, "1") == 0 && !any_ep(env);
    bool persist_fits = true;
    PD_TRY(gate_prepare(env, F));
    for (int64_t s = 0; s < nsteps;) {
        if (persist && persist_fits && F.gitems_h.empty() && nsteps - 1 - s >= 8) {
            const int64_t m = flip_free_run(env, std::min<int64_t>(nsteps - 1 - s, 1 << 20));
            if (m >= 8) {
                bool done = false;
                prof_begin(env, st);
                if (lps) PD_TRY((persist_any<R, true>(env, F, (int)m, &done)));
                else PD_TRY((persist_any<R, false>(env, F, (int)m, &done)));
                if (done) {
                    prof_end(env, st, m);
                    s += m;
                    continue;
                }
                prof_end(env, st, 0);
                persist_fits = false;
            }
        }
        if (graphs && nsteps - 1 - s >= kGraphSteps && flip_free_steps(env, kGraphSteps)) {
            PD_TRY(poll_gate_flags(env, F, blocking));
            prof_begin(env, st);
            PD_TRY(replay_graph(env, F, lps));
            prof_end(env, st, kGraphSteps);
            s += kGraphSteps;
            continue;
        }
        const bool last = s == nsteps - 1;
        // a ScaleFixWait check! after this step's velocity BC ends the
        // fused step there (MODE 2/4), scales, and restarts with a prologue
        const bool check = scale_check_due(env);
        const bool stop = last || check;
        StepArgs<R> a = args(env, F);
        a.dir_vel = dir_bits(env);
        advance_bc_clock(env);
        a.dir_pos = dir_bits(env);
        a.ts = env->ts;
        gate_launch(env, a, F);
        if (!F.gitems_h.empty()) ++F.gate_runs;
        if (!contacts) prof_begin(env, st);
        if (lps) launch_theta(st, wps, a);
        if (a.ep) launch_td(st, wps, a);
        if (!contacts) {
            if (stop) launch_step<R, 2>(st, wps, a);
            else launch_step<R, 1>(st, wps, a);
            prof_end(env, st);
        } else {
            // contact accelerations at this step's positions into F.cacc,
            // then the fused step adds them before integrating
            StepArgs<R> b = a;
            b.f = F.cacc.p;
            PD_TRY(contacts_fast(env, b));
            a.cacc = F.cacc.p;
            prof_begin(env, st);
            if (stop) launch_step<R, 2>(st, wps, a);
            else launch_step<R, 1>(st, wps, a);
            prof_end(env, st);
            contacts_clear(env, F.cacc.p);
        }
        if (a.ep) env->ecur = 1 - env->ecur;
        if (check) {
            for (size_t k = 0; k < env->hbc.size(); ++k) {
                if (!env->hbc[k].scales_at(env->ts - 1)) continue;
                const int64_t sn = env->bcs[k].sn, n = env->bcs[k].n;
                if (sn > 0) {
                    k_fscale<R><<<gridn(sn, 256), 256, 0, st>>>(a, (int)k);
                    note_launch();
                }
                if (n > 0) {
                    k_fsnapshot<R><<<gridn(n, 256), 256, 0, st>>>(a, (int)k);
                    note_launch();
                }
            }
            if (!last) {
                StepArgs<R> b = args(env, F);
                b.dir_pos = dir_bits(env);
                k_prologue<R><<<grid, kT, 0, st>>>(b);
                note_launch();
                F.cur = 1 - F.cur;
            }
        } else if (!last) {
            F.cur = 1 - F.cur;
        }
        if ((s & 63) == 63) CK(cudaGetLastError());
        ++s;
    }
    CK(cudaGetLastError());
    if (blocking && F.flags_pending) {  // land the last read-back before the state can be reset
        CK(cudaEventSynchronize(F.flags_ev));
        for (size_t b = 0; b < env->hb.size(); ++b)
            if (F.flags_h[b]) env->deformed_h[b] = 1;
        F.flags_pending = false;
    }
    return PD_OK;
}

template <class R>
pd_status update_acc_fast(pd_env *env, Fast<R> &F) {
    PD_TRY(autotune(env, F));
    StepArgs<R> a = args(env, F);
    PD_TRY(gate_if_needed(env, a, F));
    prof_begin(env, env->st);
    if (need_theta(env)) launch_theta(env->st, F.wps, a);
    if (a.ep) launch_td(env->st, F.wps, a);
    launch_step<R, 0>(env->st, F.wps, a);
    prof_end(env, env->st);
    if (a.ep) env->ecur = 1 - env->ecur;
    PD_TRY(contacts_fast(env, a));
    return PD_OK;
}

template <class R>
pd_status export_fast(pd_env *env, Fast<R> &F) {
    StepArgs<R> a = args(env, F);
    k_export<R><<<gridn(env->N, 256), 256, 0, env->st>>>(env->N, env->x4.p, env->y.p, env->v.p, env->f.p, env->p.p,
                                                         env->mth.p, a);
    note_launch();
    CK(cudaGetLastError());
    return PD_OK;
}

pd_status ensure_fast(pd_env *env) {
    if (any_ep(env) && env->nnz >= ((int64_t)1 << 31))
        return fail(PD_ERR_UNSUPPORTED, "elasto-plastic throughput mode: more than 2^31 bond slots");
    if (env->hbc.size() > (size_t)kMaxFastBC)
        return fail(PD_ERR_UNSUPPORTED, "the throughput modes support at most %d boundary conditions", kMaxFastBC);
    if (!env->fast) {
        FastHolder *h = new (std::nothrow) FastHolder();
        if (!h) return fail(PD_ERR_OOM, "host allocation failed");
        h->prec = env->precision;
        env->fast = h;
    }
    FastHolder *h = holder(env);
    if (!env->fast_valid) {
        if (h->prec == PD_PREC_FP32C) PD_TRY(init_fast(env, h->f32));
        else PD_TRY(init_fast(env, h->f64));
        env->fast_valid = true;
        h->dirty = false;
    }
    return PD_OK;
}

pd_status refresh_deformed_flags(pd_env *env) {
    bool all = true;
    for (size_t b = 0; b < env->hb.size(); ++b)
        if (env->hb[b].kind != PD_MAT_SKIP && !env->deformed_h[b]) all = false;
    if (all) return PD_OK;
    std::vector<int32_t> h(env->hb.size());
    CK(cudaMemcpyAsync(h.data(), env->deformed.p, h.size() * 4, cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    for (size_t b = 0; b < h.size(); ++b) env->deformed_h[b] = h[b];
    return PD_OK;
}

}  // namespace

pd_status sync_state_to_fp64(pd_env *env, bool invalidate) {
    FastHolder *h = holder(env);
    if (h && env->fast_valid && h->dirty) {
        if (h->prec == PD_PREC_FP32C) PD_TRY(export_fast(env, h->f32));
        else PD_TRY(export_fast(env, h->f64));
        CK(cudaStreamSynchronize(env->st));
        h->dirty = false;
    }
    if (invalidate) env->fast_valid = false;
    return PD_OK;
}

// Enqueue nsteps on the environment's stream without waiting for them
// (serving); the host copy of the gate flags catches up on later calls.
pd_status fast_vv_enqueue(pd_env *env, int64_t nsteps) {
    if (nsteps == 0) return PD_OK;
    PD_TRY(ensure_fast(env));
    FastHolder *h = holder(env);
    if (h->prec == PD_PREC_FP32C) PD_TRY(vv_chunk(env, h->f32, nsteps, false));
    else PD_TRY(vv_chunk(env, h->f64, nsteps, false));
    h->dirty = true;
    return PD_OK;
}

namespace {

int64_t step_blocks(int wps, int64_t N) {
    const int64_t slices = (N + 31) / 32;
    const int s = wps == 1 ? Split<1>::SPB : wps == 2 ? Split<2>::SPB : 1;
    return (slices + s - 1) / s;
}

template <class R, int W>
void launch_step_jobs(cudaStream_t st, bool last, const JobTable<R> &t) {
    const unsigned grid = (unsigned)t.bstart[t.n];
    if (last) k_step_jobs<R, W, Unroll<R>::HI, 2><<<grid, Split<W>::BT, 0, st>>>(t);
    else k_step_jobs<R, W, Unroll<R>::HI, 1><<<grid, Split<W>::BT, 0, st>>>(t);
    note_launch();
}

template <class R, int W>
void launch_theta_jobs(cudaStream_t st, const JobTable<R> &t) {
    k_theta_jobs<R, W, Unroll<R>::HI><<<(unsigned)t.bstart[t.n], Split<W>::BT, 0, st>>>(t);
    note_launch();
}

template <class R>
void dispatch_jobs(cudaStream_t st, int wps, bool theta, bool last, const JobTable<R> &t) {
    switch (wps) {
        case 1: theta ? launch_theta_jobs<R, 1>(st, t) : launch_step_jobs<R, 1>(st, last, t); break;
        case 2: theta ? launch_theta_jobs<R, 2>(st, t) : launch_step_jobs<R, 2>(st, last, t); break;
        case 4: theta ? launch_theta_jobs<R, 4>(st, t) : launch_step_jobs<R, 4>(st, last, t); break;
        default: theta ? launch_theta_jobs<R, 8>(st, t) : launch_step_jobs<R, 8>(st, last, t); break;
    }
}

// nsteps velocity-Verlet steps of every environment in envs (one precision,
// all batchable) as shared launches on stream st: a prologue over all jobs,
// then per step the dilatation of the state-based jobs and the fused step of
// every job, one launch per kernel shape and kJobsPerLaunch jobs.  The steps
// are those of vv_chunk (prologue, fused steps, a last step that stops
// after the velocity half kick), so a job's numbers do not depend on its
// batch.
template <class R>
pd_status batch_chunk(pd_env *const *envs, int n_envs, int64_t nsteps, cudaStream_t st,
                      Fast<R> &(*fast_of)(pd_env *)) {
    struct Item {
        pd_env *env;
        int wps;
        bool lps;
        StepArgs<R> a[3];  // prologue, even steps, odd steps
    };
    std::vector<Item> items(n_envs);
    for (int k = 0; k < n_envs; ++k) {
        pd_env *env = envs[k];
        Fast<R> &F = fast_of(env);
        Item &it = items[k];
        it.env = env;
        it.wps = F.wps % 100 / 10;
        it.lps = need_theta(env);
        const int c0 = F.cur;
        for (int t = 0; t < 3; ++t) {
            F.cur = t == 1 ? 1 - c0 : c0;
            it.a[t] = args(env, F);
            it.a[t].swz_g = 0;  // block b of a job walks its slice group b
            it.a[t].dir_vel = it.a[t].dir_pos = dir_bits(env);
            it.a[t].ts = 0;
        }
        F.cur = c0;
    }
    // launches: runs of up to kJobsPerLaunch jobs of one kernel shape,
    // state-based jobs first (the dilatation launches cover them only)
    std::stable_sort(items.begin(), items.end(), [](const Item &x, const Item &y) {
        return x.wps != y.wps ? x.wps < y.wps : (x.lps && !y.lps);
    });
    struct Run {
        int first, n, wps;
        bool lps;
    };
    std::vector<Run> runs;
    for (int k = 0; k < n_envs;) {
        int e = k;
        while (e < n_envs && e - k < kJobsPerLaunch && items[e].wps == items[k].wps && items[e].lps == items[k].lps)
            ++e;
        runs.push_back(Run{k, e - k, items[k].wps, items[k].lps});
        k = e;
    }
    // one table per (run, argument set); blocks per job: the kernel's grid
    auto table = [&](const Run &r, int t, bool particles) {
        JobTable<R> tab;
        std::memset(&tab, 0, sizeof(tab));
        int64_t tot = 0;
        for (int k = 0; k < r.n; ++k) {
            const Item &it = items[r.first + k];
            tab.a[k] = it.a[t];
            tab.bstart[k] = (int32_t)tot;
            tot += particles ? (int64_t)gridn(it.env->N) : step_blocks(it.wps, it.env->N);
        }
        tab.bstart[r.n] = (int32_t)tot;
        tab.n = r.n;
        return tab;
    };
    std::vector<JobTable<R>> pro, even, odd;
    for (const Run &r : runs) {
        pro.push_back(table(r, 0, true));
        even.push_back(table(r, 1, false));
        odd.push_back(table(r, 2, false));
    }
    for (const auto &t : pro) {
        k_prologue_jobs<R><<<(unsigned)t.bstart[t.n], kT, 0, st>>>(t);
        note_launch();
    }
    for (int64_t s = 0; s < nsteps; ++s) {
        const auto &tabs = (s & 1) ? odd : even;
        const bool last = s == nsteps - 1;
        for (size_t r = 0; r < runs.size(); ++r)
            if (runs[r].lps) dispatch_jobs<R>(st, runs[r].wps, true, last, tabs[r]);
        for (size_t r = 0; r < runs.size(); ++r) dispatch_jobs<R>(st, runs[r].wps, false, last, tabs[r]);
        if ((s & 63) == 63) CK(cudaGetLastError());
    }
    CK(cudaGetLastError());
    // host bookkeeping, as vv_chunk leaves it: the prologue and every step
    // but the last flip the record buffers
    for (Item &it : items) {
        Fast<R> &F = fast_of(it.env);
        if (nsteps & 1) F.cur = 1 - F.cur;
        for (int64_t s = 0; s < nsteps; ++s) advance_bc_clock(it.env);
        holder(it.env)->dirty = true;
    }
    return PD_OK;
}

Fast<float> &fast32(pd_env *env) { return holder(env)->f32; }
Fast<double> &fast64(pd_env *env) { return holder(env)->f64; }

}  // namespace

// An environment the serving loop may advance in shared launches: a
// throughput precision, at most kBatchMaxParticles particles (larger jobs
// fill the device with launches of their own), every block past the
// deformed gate (known on the host), no contacts, no boundary conditions,
// no elasto-plastic blocks, and a kernel shape with the larger unroll and
// no record staging.
constexpr int64_t kBatchMaxParticles = 65536;
bool fast_batchable(pd_env *env) {
    if (env->precision == PD_PREC_FP64_SERIAL || !env->hc.empty() || !env->hbc.empty() || any_ep(env) ||
        env->N > kBatchMaxParticles)
        return false;
    for (size_t b = 0; b < env->hb.size(); ++b)
        if (env->hb[b].kind != PD_MAT_SKIP && !env->deformed_h[b]) return false;
    if (ensure_fast(env) != PD_OK) return false;
    FastHolder *h = holder(env);
    const int w = h->prec == PD_PREC_FP32C ? h->f32.wps : h->f64.wps;
    const int u = h->prec == PD_PREC_FP32C ? Unroll<float>::HI : Unroll<double>::HI;
    return w > 0 && w < 100 && w % 10 == u;
}

// Shared-launch chunk of nsteps steps over envs (all batchable, one
// precision) on stream st.
pd_status fast_batch_steps(pd_env *const *envs, int n_envs, int64_t nsteps, cudaStream_t st) {
    if (n_envs <= 0 || nsteps <= 0) return PD_OK;
    const int prec = envs[0]->precision;
    for (int k = 0; k < n_envs; ++k)
        if (envs[k]->precision != prec || !envs[k]->fast_valid)
            return fail(PD_ERR_ARG, "a batch holds prepared environments of one precision");
    if (prec == PD_PREC_FP32C) return batch_chunk<float>(envs, n_envs, nsteps, st, fast32);
    return batch_chunk<double>(envs, n_envs, nsteps, st, fast64);
}

// Wait for and apply an outstanding gate-flag read-back (before anything
// resets the flags).
pd_status fast_land_flags(pd_env *env) {
    if (!env->fast) return PD_OK;
    FastHolder *h = holder(env);
    auto land = [&](auto &F) -> pd_status {
        if (!F.flags_pending) return PD_OK;
        CK(cudaEventSynchronize(F.flags_ev));
        for (size_t b = 0; b < env->hb.size(); ++b)
            if (F.flags_h[b]) env->deformed_h[b] = 1;
        F.flags_pending = false;
        return PD_OK;
    };
    return h->prec == PD_PREC_FP32C ? land(h->f32) : land(h->f64);
}

void fast_release(pd_env *env) {
    delete holder(env);
    env->fast = nullptr;
    env->fast_valid = false;
}

// A persistent chunk whose grid barrier gave up (blocks not co-resident)
// leaves its error flag set: report it and clear it.
pd_status persist_check(pd_env *env) {
    FastHolder *h = holder(env);
    auto chk = [&](auto &F) -> pd_status {
        if (!F.persisted) return PD_OK;
        F.persisted = false;
        GridBar gb;
        CK(cudaMemcpy(&gb, F.gbar.p, sizeof(gb), cudaMemcpyDeviceToHost));
        if (gb.err) {
            CK(cudaMemset(F.gbar.p, 0, sizeof(GridBar)));
            return fail(PD_ERR_TIMEOUT, "persistent step kernel: grid barrier timed out");
        }
        return PD_OK;
    };
    return h->prec == PD_PREC_FP32C ? chk(h->f32) : chk(h->f64);
}

// A staged kernel whose staging copies timed out fell back to global loads
// (results unaffected) and raised the flag: report it.
pd_status stage_check(pd_env *env) {
    FastHolder *h = holder(env);
    if (h->prec != PD_PREC_FP32C || h->f32.wps < 100 || !h->f32.serr.p) return PD_OK;
    int32_t e = 0;
    CK(cudaMemcpy(&e, h->f32.serr.p, sizeof(e), cudaMemcpyDeviceToHost));
    if (e) {
        CK(cudaMemset(h->f32.serr.p, 0, sizeof(e)));
        return fail(PD_ERR_TIMEOUT, "staged step kernel: a record staging copy did not complete in time");
    }
    return PD_OK;
}

pd_status fast_vv_steps(pd_env *env, int64_t nsteps) {
    if (nsteps == 0) return PD_OK;
    PD_TRY(ensure_fast(env));
    FastHolder *h = holder(env);
    if (h->prec == PD_PREC_FP32C) PD_TRY(vv_chunk(env, h->f32, nsteps));
    else PD_TRY(vv_chunk(env, h->f64, nsteps));
    h->dirty = true;
    PD_TRY(refresh_deformed_flags(env));
    CK(cudaStreamSynchronize(env->st));
    PD_TRY(stage_check(env));
    return persist_check(env);
}

pd_status fast_update_acc(pd_env *env) {
    PD_TRY(ensure_fast(env));
    FastHolder *h = holder(env);
    if (h->prec == PD_PREC_FP32C) PD_TRY(update_acc_fast(env, h->f32));
    else PD_TRY(update_acc_fast(env, h->f64));
    h->dirty = true;
    PD_TRY(refresh_deformed_flags(env));
    CK(cudaStreamSynchronize(env->st));
    return PD_OK;
}

}  // namespace pd

extern "C" pd_status pd_env_set_kernel_shape(pd_env *env, int32_t warps_per_slice, int32_t unroll) {
    if (!env) return pd::fail(PD_ERR_ARG, "environment handle is NULL");
    const int lo = env->precision == PD_PREC_FP32C ? pd::Unroll<float>::LO : pd::Unroll<double>::LO;
    const int hi = env->precision == PD_PREC_FP32C ? pd::Unroll<float>::HI : pd::Unroll<double>::HI;
    const int w = warps_per_slice, u = unroll;
    if (!(w == 0 && u == 0) && !((w == 1 || w == 2 || w == 4 || w == 8) && (u == lo || u == hi)))
        return pd::fail(PD_ERR_ARG, "kernel shape (%d, %d) not available: warps per slice 1/2/4/8, unroll %d or %d", w,
                    u, lo, hi);
    env->shape = w == 0 ? 0 : 10 * w + u;
    if (env->fast) {
        pd::holder(env)->f32.wps = 0;
        pd::holder(env)->f64.wps = 0;
    }
    return PD_OK;
}

extern "C" pd_status pd_env_kernel_shape(pd_env *env, int32_t *warps_per_slice, int32_t *unroll) {
    if (!env || !warps_per_slice || !unroll) return pd::fail(PD_ERR_ARG, "NULL argument");
    int cfg = 0;
    if (env->fast) cfg = env->precision == PD_PREC_FP32C ? pd::holder(env)->f32.wps : pd::holder(env)->f64.wps;
    *warps_per_slice = cfg % 100 / 10;
    *unroll = cfg % 10;
    return PD_OK;
}

extern "C" pd_status pd_env_set_record_staging(pd_env *env, int32_t mode) {
    if (!env) return pd::fail(PD_ERR_ARG, "environment handle is NULL");
    if (mode < 0 || mode > 2) return pd::fail(PD_ERR_ARG, "record staging mode %d: use 0, 1 or 2", mode);
    env->staging = mode;
    if (env->fast) {
        pd::holder(env)->f32.wps = 0;
        pd::holder(env)->f64.wps = 0;
    }
    return PD_OK;
}

extern "C" pd_status pd_env_record_staging(pd_env *env, int32_t *staged, int64_t *slices, int64_t *max_records) {
    if (!env) return pd::fail(PD_ERR_ARG, "environment handle is NULL");
    int cfg = 0;
    if (env->fast && env->precision == PD_PREC_FP32C) cfg = pd::holder(env)->f32.wps;
    if (staged) *staged = cfg >= 100;
    if (slices) *slices = env->splan_slices;
    if (max_records) *max_records = env->splan_max;
    return PD_OK;
}

// ---------------------------------------------------------------------
// Halo exchange of a slab decomposition (peridyn_b200/slabs.py): the live
// state of listed particles packed as 9 doubles each -- q (the position y
// in the serial mode, the FP64 displacement u in the throughput modes,
// which the receiving slab holds in the same form), velocity, force --
// and unpacked into another environment's particles.  Copies of the same
// numbers, so a ghost continues exactly as its owner.
// ---------------------------------------------------------------------
namespace pd {
namespace {

template <class R>
__global__ void k_pack_fast(StepArgs<R> a, const int64_t *map, const int64_t *idx, int64_t n, double *buf) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t p = map[idx[i]];
    double u0, u1, u2;
    load_u(a, p, u0, u1, u2);
    const typename Tr<R>::V4 v = a.v[p], f = a.f[p];
    double *o = buf + 9 * i;
    o[0] = u0, o[1] = u1, o[2] = u2;
    o[3] = (double)v.x, o[4] = (double)v.y, o[5] = (double)v.z;
    o[6] = (double)f.x, o[7] = (double)f.y, o[8] = (double)f.z;
}

template <class R>
__global__ void k_unpack_fast(StepArgs<R> a, const int64_t *map, const int64_t *idx, int64_t n, const double *buf) {
    using V4 = typename Tr<R>::V4;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t p = map[idx[i]];
    const double *o = buf + 9 * i;
    if (sizeof(R) == 4) {  // FP32C: the FP64 accumulator is the state; records follow at the next step
        a.ax[p] = o[0];
        a.ay[p] = o[1];
        a.az[p] = o[2];
    } else {  // FP64: the current record holds u
        V4 *cur = const_cast<V4 *>(a.xu);
        cur[2 * p + 1] = V4{(R)o[0], (R)o[1], (R)o[2], cur[2 * p].w};
    }
    a.v[p] = V4{(R)o[3], (R)o[4], (R)o[5], R(0)};
    a.f[p] = V4{(R)o[6], (R)o[7], (R)o[8], R(0)};
}

__global__ void k_pack_fp64(const double4 *y, const double4 *v, const double4 *f, const int64_t *map,
                            const int64_t *idx, int64_t n, double *buf) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t p = map[idx[i]];
    const double4 a = y[p], b = v[p], c = f[p];
    double *o = buf + 9 * i;
    o[0] = a.x, o[1] = a.y, o[2] = a.z, o[3] = b.x, o[4] = b.y, o[5] = b.z, o[6] = c.x, o[7] = c.y, o[8] = c.z;
}

__global__ void k_unpack_fp64(double4 *y, double4 *v, double4 *f, const int64_t *map, const int64_t *idx, int64_t n,
                              const double *buf) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t p = map[idx[i]];
    const double *o = buf + 9 * i;
    y[p] = make_double4(o[0], o[1], o[2], 0.0);
    v[p] = make_double4(o[3], o[4], o[5], 0.0);
    f[p] = make_double4(o[6], o[7], o[8], 0.0);
}

pd_status halo_check(pd_env *env, const int64_t *idx, int64_t n, const void *buf) {
    if (!env) return fail(PD_ERR_ARG, "environment handle is NULL");
    if (!env->finalized) return fail(PD_ERR_STATE, "environment is not finalized (call pd_env_finalize)");
    if (n < 0) return fail(PD_ERR_ARG, "n < 0");
    if (n > 0 && (!idx || !buf)) return fail(PD_ERR_ARG, "idx or buf is NULL");
    CK(cudaSetDevice(env->device));
    return PD_OK;
}

}  // namespace
}  // namespace pd

extern "C" pd_status pd_env_pack_halo(pd_env *env, const int64_t *idx, int64_t n, double *buf) {
    using namespace pd;
    PD_TRY(halo_check(env, idx, n, buf));
    if (n == 0) return PD_OK;
    FastHolder *h = holder(env);
    const unsigned g = gridn(n, 256);
    if (h && env->fast_valid) {
        if (h->prec == PD_PREC_FP32C)
            k_pack_fast<float><<<g, 256, 0, env->st>>>(args(env, h->f32), env->map.p, idx, n, buf);
        else
            k_pack_fast<double><<<g, 256, 0, env->st>>>(args(env, h->f64), env->map.p, idx, n, buf);
    } else {
        k_pack_fp64<<<g, 256, 0, env->st>>>(env->y.p, env->v.p, env->f.p, env->map.p, idx, n, buf);
    }
    note_launch();
    CK(cudaGetLastError());
    return PD_OK;
}

extern "C" pd_status pd_env_unpack_halo(pd_env *env, const int64_t *idx, int64_t n, const double *buf) {
    using namespace pd;
    PD_TRY(halo_check(env, idx, n, buf));
    if (n == 0) return PD_OK;
    FastHolder *h = holder(env);
    const unsigned g = gridn(n, 256);
    if (h && env->fast_valid) {
        if (h->prec == PD_PREC_FP32C)
            k_unpack_fast<float><<<g, 256, 0, env->st>>>(args(env, h->f32), env->map.p, idx, n, buf);
        else
            k_unpack_fast<double><<<g, 256, 0, env->st>>>(args(env, h->f64), env->map.p, idx, n, buf);
        h->dirty = true;  // the throughput state is now newer than the FP64 arrays
    } else {
        k_unpack_fp64<<<g, 256, 0, env->st>>>(env->y.p, env->v.p, env->f.p, env->map.p, idx, n, buf);
    }
    note_launch();
    CK(cudaGetLastError());
    return PD_OK;
}
