// pd_exact.cu -- FP64 kernels whose results must be bit-identical to the
// reference's CPU path.  This translation unit is compiled with
// -fmad=false: every a*b+c below rounds twice, exactly like Julia's
// unfused Float64 arithmetic.  Division and sqrt on double are IEEE
// round-to-nearest in CUDA.
//
// Expression order follows the reference literally:
//   get_magnitude  sqrt(a1*a1 + a2*a2 + a3*a3)        const_macros.jl:116
//   get_ij         x[:, j] - x[:, i]                   const_macros.jl:153-155
//   stretch        (|Y| - |X|) / |X|                   general_material.jl:338-341
//   force          ((0.5*t/|Y|) * Y_d * V_j) / rho_i   general_material.jl:351-362
#include <climits>
#include <cstdio>

#include "pd_internal.h"

namespace pd {

namespace {

constexpr int kThreads = 128;

inline unsigned grid_for(int64_t n, int threads = kThreads) {
    int64_t g = (n + threads - 1) / threads;
    return (unsigned)(g > 0 ? g : 1);
}

__device__ __forceinline__ double mag3(double a1, double a2, double a3) {
    return sqrt(a1 * a1 + a2 * a2 + a3 * a3);
}

__device__ __forceinline__ int64_t sell_base(const int64_t *slice_ptr, int64_t p) {
    return slice_ptr[p >> 5] + (p & 31);
}
__device__ __forceinline__ int64_t word_base(const int64_t *slice_ptr, int64_t p) {
    return (slice_ptr[p >> 5] >> 5) + (p & 31);
}

// ---------------------------------------------------------------------
// Family build (peri.jl:533-576): membership is the reference's exact
// test ((a1-a2)^2 + (b1-b2)^2) + (c1-c2)^2 < h*h over the 27 cells around
// the particle's cell (cells are at least one horizon wide, so the search
// is complete); the list is then sorted descending (sort + reverse,
// peri.jl:553-556 and general_material.jl:88-90).
// ---------------------------------------------------------------------
template <bool kFill>
__global__ void k_neighbors(int64_t n, int64_t first, const double4 *__restrict__ x4,
                            const int32_t *__restrict__ cell_of,
                            const int32_t *__restrict__ cell_start,
                            const int32_t *__restrict__ cell_list, int64_t cell_base, int3 dims,
                            double horizon, int32_t *__restrict__ cnt,
                            const int64_t *__restrict__ slice_ptr, int32_t *__restrict__ nbr) {
    int64_t li = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (li >= n) return;
    int64_t i = first + li;
    double4 xi = x4[i];
    int32_t c = cell_of[li] - (int32_t)cell_base;
    int cx = c % dims.x, cy = (c / dims.x) % dims.y, cz = c / (dims.x * dims.y);
    const double h2 = horizon * horizon;
    int32_t k = 0;
    int64_t base = kFill ? sell_base(slice_ptr, i) : 0;
    for (int dz = -1; dz <= 1; ++dz) {
        int zz = cz + dz;
        if (zz < 0 || zz >= dims.z) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            int yy = cy + dy;
            if (yy < 0 || yy >= dims.y) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                int xx = cx + dx;
                if (xx < 0 || xx >= dims.x) continue;
                int64_t cell = cell_base + xx + (int64_t)dims.x * (yy + (int64_t)dims.y * zz);
                for (int32_t s = cell_start[cell]; s < cell_start[cell + 1]; ++s) {
                    int32_t j = cell_list[s];
                    if (j == i) continue;
                    double4 xj = x4[j];
                    double a = xi.x - xj.x, b = xi.y - xj.y, cc = xi.z - xj.z;
                    if (a * a + b * b + cc * cc < h2) {
                        if (kFill) nbr[base + 32 * (int64_t)k] = j;
                        ++k;
                    }
                }
            }
        }
    }
    if (!kFill) cnt[i] = k;
}

// Cell binning of one block for the family search (a counting sort by cell
// id on the device): the cell of particle i is floor((x - lo) / cell) per
// axis, clamped to the grid (wider domains fold into the edge cells), as
// an index into the environment's concatenated cell grids; k_cell_ids
// counts the particles of each cell, the host turns the counts into cell
// starts, k_cell_scatter fills each cell's list.  The order within a cell
// is whatever the atomics give: the search finds the same members in any
// order and sorts each list afterwards.
__global__ void k_cell_ids(int64_t n, int64_t first, const double4 *__restrict__ x4, double3 lo, double cell,
                           int3 dims, int64_t cell_base, int32_t *__restrict__ cell_of, int32_t *__restrict__ count) {
    const int64_t li = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (li >= n) return;
    const double4 x = x4[first + li];
    const double xs[3] = {x.x, x.y, x.z}, los[3] = {lo.x, lo.y, lo.z};
    const int dm[3] = {dims.x, dims.y, dims.z};
    int ijk[3];
    for (int d = 0; d < 3; ++d) {
        double q = floor((xs[d] - los[d]) / cell);
        if (!(q >= 0.0)) q = 0.0;
        if (q > dm[d] - 1) q = dm[d] - 1;
        ijk[d] = (int)q;
    }
    const int64_t c = cell_base + ijk[0] + (int64_t)dm[0] * (ijk[1] + (int64_t)dm[1] * ijk[2]);
    cell_of[li] = (int32_t)c;
    atomicAdd(count + c, 1);
}

__global__ void k_cell_scatter(int64_t n, int64_t first, const int32_t *__restrict__ cell_of,
                               int32_t *__restrict__ cursor, int32_t *__restrict__ cell_list) {
    const int64_t li = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (li >= n) return;
    cell_list[atomicAdd(cursor + cell_of[li], 1)] = (int32_t)(first + li);
}

// Insertion sort of one particle's strided list into descending order.
__global__ void k_sort_neighbors(int64_t N, const int64_t *__restrict__ slice_ptr,
                                 const int32_t *__restrict__ cnt, int32_t *__restrict__ nbr) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= N) return;
    int32_t n = cnt[p];
    int32_t *a = nbr + sell_base(slice_ptr, p);
    for (int32_t k = 1; k < n; ++k) {
        int32_t v = a[32 * (int64_t)k];
        int32_t j = k - 1;
        while (j >= 0 && a[32 * (int64_t)j] < v) {
            a[32 * (int64_t)(j + 1)] = a[32 * (int64_t)j];
            --j;
        }
        a[32 * (int64_t)(j + 1)] = v;
    }
}

__global__ void k_init_intact(int64_t N, const int64_t *__restrict__ slice_ptr,
                              const int32_t *__restrict__ cnt, uint32_t *__restrict__ words) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= N) return;
    int32_t n = cnt[p];
    int64_t wb = word_base(slice_ptr, p);
    for (int32_t w = 0; w * 32 < n; ++w) {
        int32_t rem = n - w * 32;
        words[wb + 32 * (int64_t)w] = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
    }
}

// ---------------------------------------------------------------------
// Runtime layout on the device (the conversion build_runtime_layout in
// pd_env.cu performs on the host; both give the same arrays).  Pass 1, one
// warp per slice: the union of the lanes' neighbour offsets q - p, merged
// from the lanes' descending lists one element at a time (the warp's
// maximum of the lanes' heads is the union's next element; lanes holding it
// advance).  A slice takes the stencil form when the union has at most
// maxc + maxc/4 + 32 entries (maxc: the slice's largest family) and every
// union offset of every lane with bonds names an in-range record.
// Outputs per slice: mode, union length (stencil) and the union itself in
// uni[s * ustride ...]; the first merge only counts, so a slice found too
// large writes nothing.
// ---------------------------------------------------------------------
__global__ void k_layout_union(int64_t S, int64_t N, const int64_t *__restrict__ slice_ptr,
                               const int32_t *__restrict__ cnt, const int32_t *__restrict__ nbr_b,
                               int32_t force_explicit, int64_t ustride, int32_t *__restrict__ mode,
                               int32_t *__restrict__ len, int32_t *__restrict__ uni) {
    const int64_t s = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= S) return;  // whole warps: blockDim is a multiple of 32
    const int64_t p = s * 32 + lane;
    const int32_t c = cnt[p];
    int32_t maxc = c;
    for (int o = 16; o > 0; o >>= 1) maxc = max(maxc, __shfl_xor_sync(0xffffffffu, maxc, o));
    const int32_t *lst = nbr_b + slice_ptr[s] + lane;  // lane's k-th neighbour at lst[32 k]
    const int64_t limit = (int64_t)maxc + maxc / 4 + 32;
    bool stencil = !force_explicit && maxc > 0;
    int64_t ulen = 0;
    int32_t umax = 0, umin = 0;
    if (stencil) {
        for (int pass = 0; pass < 2 && stencil; ++pass) {
            int32_t k = 0;
            int32_t head = k < c ? lst[0] - (int32_t)p : INT_MIN;
            int64_t pos = 0;
            for (;;) {
                const int32_t m = __reduce_max_sync(0xffffffffu, head);
                if (m == INT_MIN) break;
                if (pass == 0) {
                    if (pos == 0) umax = m;
                    umin = m;
                    if (pos + 1 > limit) {
                        stencil = false;
                        break;
                    }
                } else if (lane == 0) {
                    uni[s * ustride + pos] = m;
                }
                if (head == m) {
                    ++k;
                    head = k < c ? lst[32 * (int64_t)k] - (int32_t)p : INT_MIN;
                }
                ++pos;
            }
            ulen = pos;
            if (pass == 0 && stencil) {
                // every slot a lane scans must name an in-range record
                const bool ok = c == 0 || (p + umax < N && p + umin >= 0);
                stencil = __all_sync(0xffffffffu, ok);
            }
        }
    }
    if (lane == 0) {
        mode[s] = stencil ? kStencil : kExplicit;
        len[s] = stencil ? (int32_t)ulen : maxc;
    }
}

// Pass 2, one thread per particle (a warp per slice): the runtime arrays.
// Stencil slices: the union offsets into nbr, and each bond's slot found by
// a binary search of its offset in the (descending) union; explicit slices:
// the build layout's indices copied.  Intact and family-member bits go to
// the lane's own words; cnt_rt = last occupied slot + 1.
__global__ void k_layout_fill(int64_t N, const int64_t *__restrict__ slice_ptr, const int32_t *__restrict__ cnt,
                              const int32_t *__restrict__ nbr_b, const uint32_t *__restrict__ w_b,
                              const SliceInfo *__restrict__ si, const int32_t *__restrict__ ulen, int64_t ustride,
                              const int32_t *__restrict__ uni, int32_t *__restrict__ nbr, uint32_t *__restrict__ words,
                              uint32_t *__restrict__ fam, int32_t *__restrict__ cnt_rt) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= N) return;
    const int64_t s = p >> 5;
    const int lane = (int)(p & 31);
    const SliceInfo d = si[s];
    const int32_t c = cnt[p];
    const int64_t base = slice_ptr[s] + lane, wb = slice_ptr[s] / 32 + lane, ow = d.word + lane;
    const int32_t *u = uni + s * ustride;
    const int32_t ul = d.mode == kStencil ? ulen[s] : 0;
    if (d.mode == kStencil) {
        for (int32_t j = lane; j < ul; j += 32) nbr[d.nbr + j] = u[j];
    } else {
        for (int32_t k = 0; k < d.len; ++k) nbr[d.nbr + 32 * (int64_t)k + lane] = nbr_b[base + 32 * (int64_t)k];
    }
    int32_t last = -1;
    for (int32_t k = 0; k < c; ++k) {
        int32_t slot = k;
        if (d.mode == kStencil) {
            const int32_t o = nbr_b[base + 32 * (int64_t)k] - (int32_t)p;
            int32_t lo = 0, hi = ul - 1;  // u descends: find u[slot] == o
            while (lo < hi) {
                const int32_t mid = (lo + hi) >> 1;
                if (u[mid] > o) lo = mid + 1;
                else hi = mid;
            }
            slot = lo;
        }
        const uint32_t bit = 1u << (slot & 31);
        fam[ow + 32 * (int64_t)(slot >> 5)] |= bit;
        if ((w_b[wb + 32 * (int64_t)(k >> 5)] >> (k & 31)) & 1u) words[ow + 32 * (int64_t)(slot >> 5)] |= bit;
        last = slot;
    }
    cnt_rt[p] = last + 1;
}

__global__ void k_popcount(int64_t N, const SliceInfo *__restrict__ si,
                           const int32_t *__restrict__ cnt, const uint32_t *__restrict__ words,
                           int32_t *__restrict__ out) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= N) return;
    int32_t n = cnt[p], c = 0;
    const uint32_t *wp = words + si[p >> 5].word + (p & 31);
    for (int32_t w = 0; w * 32 < n; ++w) c += __popc(wp[32 * (int64_t)w]);
    out[p] = c;
}

// peri.jl:342-354 weighted_volume: m_i = sum_j ((1/|X|) * (|X|*|X|)) * 1 * V_j
// over the family (every member, intact or not) in stored (descending) order.
__global__ void k_weighted_volume(Geo g, double2 *__restrict__ mth) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= g.N) return;
    if (g.tinfo[p] < 0) return;
    double4 xp = g.x4[p];
    int32_t n = g.cnt[p];
    const BondRef br = bond_ref(g.si, g.nbr, g.fam, p);
    double acc = 0.0;
    for (int32_t k = 0; k < n; ++k) {
        if (!((*br.word(k) >> (k & 31)) & 1u)) continue;
        int32_t q = br.q(k);
        double4 xq = g.x4[q];
        double mg = mag3(xq.x - xp.x, xq.y - xp.y, xq.z - xp.z);
        double w = 1.0 / mg;
        acc = acc + w * (mg * mg) * 1.0 * xq.w;
    }
    mth[p].x = acc;
}

// ---------------------------------------------------------------------
// peri.jl:155-172 dilatation!: theta_i = sum over intact bonds, in family
// order, of (((3/m_i) * w) * |X|) * e * V_j  (horizon correction == 1).
// ---------------------------------------------------------------------
__global__ void k_theta_serial(Geo g, const double4 *__restrict__ y,
                               const uint32_t *__restrict__ win, double2 *__restrict__ mth,
                               int64_t p0, int64_t p1) {
    int64_t p = p0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= p1) return;
    int32_t ti = g.tinfo[p];
    if (ti < 0) return;
    const DevBlock &B = g.blocks[ti >> 8];
    if (B.kind != PD_MAT_ORDINARY_STATE_BASED && B.kind != PD_MAT_ELASTO_PLASTIC) return;
    double4 xp = g.x4[p], yp = y[p];
    double c_i = 3.0 / mth[p].x;
    int32_t n = g.cnt[p];
    const BondRef br = bond_ref(g.si, g.nbr, win, p);
    double th = 0.0;
    uint32_t w = 0;
    for (int32_t k = 0; k < n; ++k) {
        if ((k & 31) == 0) w = *br.word(k);
        if (!((w >> (k & 31)) & 1u)) continue;
        int32_t q = br.q(k);
        double4 xq = g.x4[q], yq = y[q];
        double xij = mag3(xq.x - xp.x, xq.y - xp.y, xq.z - xp.z);
        double yij = mag3(yq.x - yp.x, yq.y - yp.y, yq.z - yp.z);
        double e = yij - xij;
        double wi = 1.0 / xij;
        th = th + c_i * wi * xij * e * xq.w;
    }
    mth[p].y = th;
}

// One bond term seen from particle p: returns true when the bond is
// stretched below critical (s < cs) and writes the acceleration term
// ((xx*Y_d)*V_q)/rho_p.  The reference adds exactly this value to f_p in
// p's own loop, and subtracts its exact negation in q's loop
// (general_material.jl:357-362), so the same function serves both.
template <int KIND>
__device__ __forceinline__ bool bond_term(const Geo &g, const DevBlock &B, int tp,
                                          double4 xp, double4 yp, double2 mp, double rho_p,
                                          int32_t q, const double4 *__restrict__ y,
                                          const double2 *__restrict__ mth, double &t0,
                                          double &t1, double &t2) {
    double4 xq = g.x4[q], yq = y[q];
    double X1 = xq.x - xp.x, X2 = xq.y - xp.y, X3 = xq.z - xp.z;
    double Y1 = yq.x - yp.x, Y2 = yq.y - yp.y, Y3 = yq.z - yp.z;
    double yij = mag3(Y1, Y2, Y3);
    double xij = mag3(X1, X2, X3);
    double ext = yij - xij;
    double s = ext / xij;
    int tq = B.nt > 1 ? (g.tinfo[q] & 255) : 0;
    const PairParam &pp = g.pairs[B.pair_base + tp + tq * B.nt];
    if (!(s < pp.cs)) return false;
    double t;
    if (KIND == PD_MAT_BOND_BASED) {
        t = s * B.c11;  // bond_based.jl:195-197
    } else {
        // ordinary_state_based.jl:176-187 (w_ij == w_ji == 1/|X|)
        double2 mq = mth[q];
        double wij = 1.0 / xij;
        double a = wij / mp.x, b = wij / mq.x;
        t = pp.k35 * (mp.y * xij * a + mq.y * xij * b) + pp.g15 * ext * (a + b);
    }
    double xx = 0.5 * t / yij;
    t0 = xx * Y1 * xq.w / rho_p;
    t1 = xx * Y2 * xq.w / rho_p;
    t2 = xx * Y3 * xq.w / rho_p;
    return true;
}

// ---------------------------------------------------------------------
// Elasto-plastic solid (elasto_plastic.jl).  Unlike the PMB and LPS laws,
// the bond term depends on which end visits the bond: particle i's visit
// to bond slot k uses td_norm2[i] and edp[k, i] and updates edp[k, i].
// ---------------------------------------------------------------------
// Slot of neighbour p in q's family.
__device__ __forceinline__ int32_t find_slot(const Geo &g, int64_t q, int32_t p) {
    return slot_of(g.si, g.nbr, g.cnt, q, p);
}

// force_density_t_ij (elasto_plastic.jl:215-242) for the visit of i to j;
// mi, mj = (m, theta); the plastic update of edp[k, i] goes to *edp_new.
__device__ __forceinline__ double ep_t(const PairParam &pp, double xij, double ext, double2 mi, double2 mj,
                                       double td2_i, double edp_old, double *edp_new) {
    const double wij = 1.0 / xij;  // influence_function(X) == influence_function(-X)
    const double C = sqrt(pp.psi2 / td2_i);
    const double a = wij / mi.x, b = wij / mj.x;
    const double tw = mi.y * a + mj.y * b;
    const double theta_ij = tw / (a + b);
    const double ed = ext - theta_ij * xij / 3;
    const double ede = ed - edp_old;
    const double td_trial = pp.g15 * (a + b) * ede;
    double td;
    if (C > 1) {
        td = td_trial;
    } else {
        td = C * td_trial;
        if (edp_new) *edp_new = edp_old + ede * (1 - C);
    }
    const double tn = pp.k35 * xij * tw;
    return tn + td;
}

// The elasto-plastic term seen by p for the bond to q: from p's own visit
// (own, slot k of p) or from q's visit to p.
__device__ __forceinline__ bool bond_term_ep(const Geo &g, const DevBlock &B, int tp, int64_t p, double4 xp,
                                             double4 yp, double2 mp, double rho_p, int32_t q, int32_t k, bool own,
                                             const double4 *__restrict__ y, const double2 *__restrict__ mth,
                                             double &t0, double &t1, double &t2) {
    double4 xq = g.x4[q], yq = y[q];
    double X1 = xq.x - xp.x, X2 = xq.y - xp.y, X3 = xq.z - xp.z;
    double Y1 = yq.x - yp.x, Y2 = yq.y - yp.y, Y3 = yq.z - yp.z;
    double yij = mag3(Y1, Y2, Y3);
    double xij = mag3(X1, X2, X3);
    double ext = yij - xij;
    double s = ext / xij;
    int tq = B.nt > 1 ? (g.tinfo[q] & 255) : 0;
    const PairParam &pp = g.pairs[B.pair_base + tp + tq * B.nt];
    if (!(s < pp.cs)) return false;
    const double2 mq = mth[q];
    double t;
    if (own) {
        const int64_t e = slot_index(g.si, p, k);
        t = ep_t(pp, xij, ext, mp, mq, g.td2[p], g.edp_in[e], g.edp_out + e);
    } else {
        const int64_t e = slot_index(g.si, q, find_slot(g, q, (int32_t)p));
        t = ep_t(pp, xij, ext, mq, mp, g.td2[q], g.edp_in[e], nullptr);
    }
    double xx = 0.5 * t / yij;
    t0 = xx * Y1 * xq.w / rho_p;
    t1 = xx * Y2 * xq.w / rho_p;
    t2 = xx * Y3 * xq.w / rho_p;
    return true;
}

// peri.jl:411-445 loop_over_neighs! with td_norm2_ij! (elasto_plastic.jl:
// 274-288): td_norm2[p] over p's family in stored order; bonds at or beyond
// the critical stretch are cleared (that loop breaks them too).  Particles
// of other blocks only copy their flags.
__global__ void __launch_bounds__(kThreads)
    k_td_serial(Geo g, const double4 *__restrict__ y, const double2 *__restrict__ mth,
                const uint32_t *__restrict__ win, uint32_t *__restrict__ wout, int64_t p0, int64_t p1) {
    int64_t p = p0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= p1) return;
    const int32_t ti = g.tinfo[p];
    const int32_t n = g.cnt[p];
    const int64_t wb = g.si[p >> 5].word + (p & 31);
    const bool active = ti >= 0 && g.blocks[ti >> 8].kind == PD_MAT_ELASTO_PLASTIC && g.deformed[ti >> 8] != 0;
    if (!active) {
        for (int32_t w = 0; w * 32 < n; ++w) wout[wb + 32 * (int64_t)w] = win[wb + 32 * (int64_t)w];
        return;
    }
    const DevBlock &B = g.blocks[ti >> 8];
    const int tp = ti & 255;
    const double4 xp = g.x4[p], yp = y[p];
    const double2 mp = mth[p];
    const BondRef br = bond_ref(g.si, g.nbr, win, p);
    uint32_t *wo = wout + wb;
    double acc = 0.0;
    uint32_t w = 0;
    for (int32_t k = 0; k < n; ++k) {
        if ((k & 31) == 0) {
            if (k > 0) wo[32 * (int64_t)((k >> 5) - 1)] = w;
            w = *br.word(k);
        }
        if (!((w >> (k & 31)) & 1u)) continue;
        const int32_t q = br.q(k);
        const double4 xq = g.x4[q], yq = y[q];
        const double X1 = xq.x - xp.x, X2 = xq.y - xp.y, X3 = xq.z - xp.z;
        const double Y1 = yq.x - yp.x, Y2 = yq.y - yp.y, Y3 = yq.z - yp.z;
        const double yij = mag3(Y1, Y2, Y3);
        const double xij = mag3(X1, X2, X3);
        const double ext = yij - xij;
        const double s = ext / xij;
        const int tq = B.nt > 1 ? (g.tinfo[q] & 255) : 0;
        const PairParam &pp = g.pairs[B.pair_base + tp + tq * B.nt];
        if (s < pp.cs) {
            const double2 mq = mth[q];
            const double wij = 1.0 / xij;
            const double a = wij / mp.x, b = wij / mq.x;
            const double w_m = a + b;
            const double tw = mp.y * a + mq.y * b;
            const double theta_ij = tw / w_m;
            const double ed = ext - theta_ij * xij / 3;
            const double td = pp.g15 * (ed - g.edp_in[slot_index(g.si, p, k)]) * w_m;
            acc = acc + td * td * xq.w;
        } else {
            w &= ~(1u << (k & 31));
        }
    }
    if (n > 0) wo[32 * (int64_t)((n - 1) >> 5)] = w;
    g.td2[p] = acc;
}

// ---------------------------------------------------------------------
// general_material.jl:296-369 in the serial loop's summation order.
// The reference visits i = 1..N and, for each i, its family in stored
// (descending) order, adding the term to f_i and subtracting it from f_j.
// Particle p therefore receives, in order:
//   A. terms of neighbours q < p, ascending q   (from q's loop)
//   B. terms of all neighbours, descending q    (p's own loop)
//   C. terms of neighbours q > p, ascending q   (from q's loop)
// Bond flags are symmetric (both ends break in the same step because the
// stretch is the same number from both sides), so p's own flags stand in
// for q's.  Bonds with s >= cs are cleared in wout.
// ---------------------------------------------------------------------
template <int KIND>
__device__ void force_serial_particle(const Geo &g, int64_t p, int32_t ti,
                                      const double4 *__restrict__ y,
                                      const double2 *__restrict__ mth,
                                      const uint32_t *__restrict__ win,
                                      uint32_t *__restrict__ wout, double4 *__restrict__ f,
                                      int accumulate) {
    const DevBlock &B = g.blocks[ti >> 8];
    int tp = ti & 255;
    double4 xp = g.x4[p], yp = y[p];
    double2 mp = KIND != PD_MAT_BOND_BASED ? mth[p] : make_double2(0.0, 0.0);
    constexpr bool EP = KIND == PD_MAT_ELASTO_PLASTIC;
    double rho_p = g.tdens[B.type_base + tp];
    int32_t n = g.cnt[p];
    const BondRef br = bond_ref(g.si, g.nbr, win, p);
    uint32_t *wo = wout + g.si[p >> 5].word + (p & 31);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    if (accumulate) {
        double4 f0 = f[p];
        fx = f0.x;
        fy = f0.y;
        fz = f0.z;
    }
    double t0, t1, t2;
    // Pass A: q < p, ascending (walk the descending list from the end).
    int32_t k = n - 1;
    for (; k >= 0; --k) {
        int32_t q = br.q(k);
        if (q > p) break;
        uint32_t w = *br.word(k);
        if (!((w >> (k & 31)) & 1u)) continue;
        if (EP ? bond_term_ep(g, B, tp, p, xp, yp, mp, rho_p, q, k, false, y, mth, t0, t1, t2)
               : bond_term<KIND>(g, B, tp, xp, yp, mp, rho_p, q, y, mth, t0, t1, t2)) {
            fx = fx + t0;
            fy = fy + t1;
            fz = fz + t2;
        }
    }
    const int32_t kc = k;
    // Pass B: p's own loop, descending q; breaks bonds.
    uint32_t w = 0;
    for (k = 0; k < n; ++k) {
        if ((k & 31) == 0) {
            if (k > 0) wo[32 * (int64_t)((k >> 5) - 1)] = w;
            w = *br.word(k);
        }
        if (EP) {  // edp carries over unless this visit yields
            const int64_t e = slot_index(g.si, p, k);
            g.edp_out[e] = g.edp_in[e];
        }
        if (!((w >> (k & 31)) & 1u)) continue;
        int32_t q = br.q(k);
        if (EP ? bond_term_ep(g, B, tp, p, xp, yp, mp, rho_p, q, k, true, y, mth, t0, t1, t2)
               : bond_term<KIND>(g, B, tp, xp, yp, mp, rho_p, q, y, mth, t0, t1, t2)) {
            fx = fx + t0;
            fy = fy + t1;
            fz = fz + t2;
        } else {
            w &= ~(1u << (k & 31));
        }
    }
    if (n > 0) wo[32 * (int64_t)((n - 1) >> 5)] = w;
    // Pass C: q > p, ascending.
    for (k = kc; k >= 0; --k) {
        int32_t q = br.q(k);
        uint32_t ww = *br.word(k);
        if (!((ww >> (k & 31)) & 1u)) continue;
        if (EP ? bond_term_ep(g, B, tp, p, xp, yp, mp, rho_p, q, k, false, y, mth, t0, t1, t2)
               : bond_term<KIND>(g, B, tp, xp, yp, mp, rho_p, q, y, mth, t0, t1, t2)) {
            fx = fx + t0;
            fy = fy + t1;
            fz = fz + t2;
        }
    }
    f[p] = make_double4(fx, fy, fz, 0.0);
}

__global__ void __launch_bounds__(kThreads)
    k_force_serial(Geo g, const double4 *__restrict__ y, const double2 *__restrict__ mth,
                   const uint32_t *__restrict__ win, uint32_t *__restrict__ wout,
                   double4 *__restrict__ f, int accumulate, int64_t p0, int64_t p1) {
    int64_t p = p0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= p1) return;
    int32_t ti = g.tinfo[p];
    int32_t n = g.cnt[p];
    const int64_t wb = g.si[p >> 5].word + (p & 31);
    bool active = false;
    int kind = PD_MAT_SKIP;
    if (ti >= 0) {
        const DevBlock &B = g.blocks[ti >> 8];
        kind = B.kind;
        active = kind != PD_MAT_SKIP && g.deformed[ti >> 8] != 0;
    }
    if (!active) {
        for (int32_t w = 0; w * 32 < n; ++w) wout[wb + 32 * (int64_t)w] = win[wb + 32 * (int64_t)w];
        if (kind == PD_MAT_ELASTO_PLASTIC && g.edp_out)
            for (int32_t k = 0; k < n; ++k) g.edp_out[slot_index(g.si, p, k)] = g.edp_in[slot_index(g.si, p, k)];
        if (!accumulate) f[p] = make_double4(0.0, 0.0, 0.0, 0.0);
        return;
    }
    if (kind == PD_MAT_BOND_BASED)
        force_serial_particle<PD_MAT_BOND_BASED>(g, p, ti, y, mth, win, wout, f, accumulate);
    else if (kind == PD_MAT_ELASTO_PLASTIC)
        force_serial_particle<PD_MAT_ELASTO_PLASTIC>(g, p, ti, y, mth, win, wout, f, accumulate);
    else
        force_serial_particle<PD_MAT_ORDINARY_STATE_BASED>(g, p, ti, y, mth, win, wout, f,
                                                            accumulate);
}

// ---------------------------------------------------------------------
// velocity_verlet.jl:62-75: v .+= (dt/2) .* f ; y .+= dt .* v
// ---------------------------------------------------------------------
__global__ void k_kick_drift(int64_t N, double c, double dt, const double4 *__restrict__ f,
                             double4 *__restrict__ v, double4 *__restrict__ y) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    double4 fi = f[i], vi = v[i], yi = y[i];
    vi.x = vi.x + c * fi.x;
    vi.y = vi.y + c * fi.y;
    vi.z = vi.z + c * fi.z;
    yi.x = yi.x + dt * vi.x;
    yi.y = yi.y + dt * vi.y;
    yi.z = yi.z + dt * vi.z;
    v[i] = vi;
    y[i] = yi;
}

__global__ void k_kick(int64_t N, double c, const double4 *__restrict__ f,
                       double4 *__restrict__ v) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    double4 fi = f[i], vi = v[i];
    vi.x = vi.x + c * fi.x;
    vi.y = vi.y + c * fi.y;
    vi.z = vi.z + c * fi.z;
    v[i] = vi;
}

__device__ __forceinline__ double &comp(double4 &a, int d) {
    return d == 0 ? a.x : (d == 1 ? a.y : a.z);
}

// boundary_conditions.jl:107-111 with FixBC.jl:213 / ToFroBC.jl:286-289
__global__ void k_bc_pos(BCDev bc, double dt, int dir, int64_t ts, double4 *__restrict__ y) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= bc.n) return;
    int32_t i = bc.idx[j];
    double4 yi = y[i], last = bc.last[j];
    double step = dt * (double)dir;
    for (int d = 0; d < 3; ++d) {
        if (!((bc.dims >> d) & 1)) continue;
        if (bc.kind == PD_BC_FIX || bc.kind == PD_BC_SCALE_FIX_WAIT) {
            // FixBC.jl:213, ScaleFixWaitBC.jl:59 xF = (last, last)
            comp(yi, d) = comp(last, d);
        } else if (bc.kind == PD_BC_DELTA_SCALE) {
            // DeltaScaleBC.jl:52-55: (last - fix) * (1 + scale*dt*time_step) + fix
            const double g = 1.0 + (bc.scale[d] * dt) * (double)ts;
            comp(yi, d) = (comp(last, d) - bc.fix[d]) * g + bc.fix[d];
        } else {
            double nl = comp(last, d) + step * bc.rate[d];
            comp(yi, d) = nl;
            comp(last, d) = nl;
        }
    }
    y[i] = yi;
    if (bc.kind == PD_BC_TOFRO) bc.last[j] = last;
}

// boundary_conditions.jl:122-126 with FixBC.jl:214 / ToFroBC.jl:290
__global__ void k_bc_vel(BCDev bc, int dir, const double4 *__restrict__ y, double4 *__restrict__ v) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= bc.n) return;
    int32_t i = bc.idx[j];
    double4 vi = v[i];
    if (bc.kind == PD_BC_CONTAINER) {
        // ContainerBC.jl:63-68: v[dims] = 0 where y left the limits
        double4 yi = y[i];
        bool out = false;
        for (int d = 0; d < 3; ++d)
            if ((bc.dims >> d) & 1) out |= (comp(yi, d) < bc.lo[d]) || (comp(yi, d) > bc.hi[d]);
        if (!out) return;
        for (int d = 0; d < 3; ++d)
            if ((bc.dims >> d) & 1) comp(vi, d) = 0.0;
        v[i] = vi;
        return;
    }
    for (int d = 0; d < 3; ++d) {
        if (!((bc.dims >> d) & 1)) continue;
        comp(vi, d) = bc.kind == PD_BC_TOFRO ? (double)dir * bc.rate[d] : 0.0;
    }
    v[i] = vi;
}

// ScaleFixWaitBC.jl:63-68 (check!): y[dims, scalebool] = (y - fix) * sqrt(1 + 2*scale*dt) + fix
__global__ void k_bc_scale(BCDev bc, double dt, double4 *__restrict__ y) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= bc.sn) return;
    const int32_t i = bc.sidx[j];
    double4 yi = y[i];
    for (int d = 0; d < 3; ++d) {
        if (!((bc.dims >> d) & 1)) continue;
        const double g = sqrt(1.0 + (2.0 * bc.scale[d]) * dt);
        comp(yi, d) = (comp(yi, d) - bc.fix[d]) * g + bc.fix[d];
    }
    y[i] = yi;
}

// FixBC.jl:63 / ToFroBC.jl:94: BC.last .= y[dims, bool]
__global__ void k_bc_snapshot(BCDev bc, const double4 *__restrict__ y) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= bc.n) return;
    double4 yi = y[bc.idx[j]], last = bc.last[j];
    for (int d = 0; d < 3; ++d)
        if ((bc.dims >> d) & 1) comp(last, d) = comp(yi, d);
    bc.last[j] = last;
}

// solvers.jl:280-285 update_misc!: p = mass .* v
__global__ void k_momentum(int64_t N, const double *__restrict__ mass,
                           const double4 *__restrict__ v, double4 *__restrict__ p) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    double m = mass[i];
    double4 vi = v[i];
    p[i] = make_double4(m * vi.x, m * vi.y, m * vi.z, 0.0);
}

__global__ void k_zero4(int64_t N, double4 *__restrict__ a) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    a[i] = make_double4(0.0, 0.0, 0.0, 0.0);
}

// ---------------------------------------------------------------------
// Deformed gate: isapprox(y .- y[:,1] .+ x[:,1], x) with rtol = sqrt(eps)
// (general_material.jl:249).  Deterministic two-stage reduction.
// ---------------------------------------------------------------------
constexpr int kGateThreads = 256;

__global__ void __launch_bounds__(kGateThreads)
    k_gate_partial(const GateItem *__restrict__ items, int gx, const double4 *__restrict__ x4,
                   const double4 *__restrict__ y, double *__restrict__ part,
                   const int32_t *__restrict__ deformed) {
    const GateItem it = items[blockIdx.y];
    double *partials = part + 3 * ((int64_t)blockIdx.y * gx);
    if (deformed[it.block]) return;
    const int64_t first = it.first, n = it.n;
    __shared__ double sh[3][kGateThreads];
    double4 y1 = y[first], x1 = x4[first];
    double sd = 0.0, sa = 0.0, sx = 0.0;
    for (int64_t l = blockIdx.x * (int64_t)kGateThreads + threadIdx.x; l < n;
         l += (int64_t)gx * kGateThreads) {
        double4 yi = y[first + l], xi = x4[first + l];
        double a0 = (yi.x - y1.x) + x1.x, a1 = (yi.y - y1.y) + x1.y, a2 = (yi.z - y1.z) + x1.z;
        double d0 = a0 - xi.x, d1 = a1 - xi.y, d2 = a2 - xi.z;
        sd = sd + d0 * d0 + d1 * d1 + d2 * d2;
        sa = sa + a0 * a0 + a1 * a1 + a2 * a2;
        sx = sx + xi.x * xi.x + xi.y * xi.y + xi.z * xi.z;
    }
    sh[0][threadIdx.x] = sd;
    sh[1][threadIdx.x] = sa;
    sh[2][threadIdx.x] = sx;
    __syncthreads();
    for (int s = kGateThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] = sh[c][threadIdx.x] + sh[c][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; ++c) partials[3 * blockIdx.x + c] = sh[c][0];
}

__global__ void k_gate_final(const GateItem *__restrict__ items, int nitems, int gx,
                             const double *__restrict__ part, int32_t *__restrict__ deformed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nitems) return;
    int32_t *flag = deformed + items[i].block;
    if (*flag) return;
    const double *partials = part + 3 * ((int64_t)i * gx);
    double sd = 0.0, sa = 0.0, sx = 0.0;
    for (int b = 0; b < gx; ++b) {
        sd = sd + partials[3 * b];
        sa = sa + partials[3 * b + 1];
        sx = sx + partials[3 * b + 2];
    }
    double d = sqrt(sd);
    const double rtol = 0x1p-26;  // sqrt(eps(Float64))
    bool approx = isfinite(d) && d <= fmax(0.0, rtol * fmax(sqrt(sa), sqrt(sx)));
    if (!approx) *flag = 1;
}

// peri.jl:587-594 cal_damage: 1 - sum(intact) / intact0
__global__ void k_damage(int64_t N, const SliceInfo *__restrict__ si,
                         const int32_t *__restrict__ cnt, const uint32_t *__restrict__ words,
                         const int32_t *__restrict__ intact0, const int32_t *__restrict__ tinfo,
                         double *__restrict__ damage) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= N) return;
    if (tinfo[p] < 0) {
        damage[p] = 0.0;
        return;
    }
    int32_t n = cnt[p], c = 0;
    const int64_t wb = si[p >> 5].word + (p & 31);
    for (int32_t w = 0; w * 32 < n; ++w) c += __popc(words[wb + 32 * (int64_t)w]);
    damage[p] = 1.0 - (double)c / (double)intact0[p];
}

// Fixed partial-reduction width, independent of the device's SM count so
// that the summation order (and the rounding of the gate norms) is the same
// on every GPU.
constexpr int kSumBlocks = 148;
__global__ void __launch_bounds__(256)
    k_sum4_partial(int64_t N, const double4 *__restrict__ a, double *__restrict__ partials) {
    __shared__ double sh[3][256];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int64_t i = blockIdx.x * 256 + threadIdx.x; i < N; i += (int64_t)kSumBlocks * 256) {
        double4 v = a[i];
        s0 = s0 + v.x;
        s1 = s1 + v.y;
        s2 = s2 + v.z;
    }
    sh[0][threadIdx.x] = s0;
    sh[1][threadIdx.x] = s1;
    sh[2][threadIdx.x] = s2;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] = sh[c][threadIdx.x] + sh[c][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; ++c) partials[3 * blockIdx.x + c] = sh[c][0];
}

__global__ void k_sum4_final(const double *__restrict__ partials, double *__restrict__ out3) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int b = 0; b < kSumBlocks; ++b) {
        s0 = s0 + partials[3 * b];
        s1 = s1 + partials[3 * b + 1];
        s2 = s2 + partials[3 * b + 2];
    }
    out3[0] = s0;
    out3[1] = s1;
    out3[2] = s2;
}

__global__ void k_unpack3(int64_t n, const double *__restrict__ src3,
                          const int64_t *__restrict__ map, double4 *__restrict__ dst) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n) return;
    dst[map[e]] = make_double4(src3[3 * e], src3[3 * e + 1], src3[3 * e + 2], 0.0);
}

__global__ void k_pack3(int64_t n, const double4 *__restrict__ src,
                        const int64_t *__restrict__ map, double *__restrict__ dst3) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n) return;
    double4 v = src[map[e]];
    dst3[3 * e] = v.x;
    dst3[3 * e + 1] = v.y;
    dst3[3 * e + 2] = v.z;
}

__global__ void k_nonfinite(int64_t N, const double4 *__restrict__ a, int32_t *__restrict__ flag) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    double4 v = a[i];
    if (!isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z)) *flag = 1;
}

}  // namespace

// ---------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------
void launch_count_neighbors(cudaStream_t st, int64_t n, int64_t first, const double4 *x4,
                            const int32_t *cell_of, const int32_t *cell_start,
                            const int32_t *cell_list, int64_t cell_base, int3 dims,
                            double horizon, int32_t *cnt) {
    if (n <= 0) return;
    k_neighbors<false><<<grid_for(n), kThreads, 0, st>>>(n, first, x4, cell_of, cell_start,
                                                         cell_list, cell_base, dims, horizon, cnt,
                                                         nullptr, nullptr); pd::note_launch();
}

void launch_fill_neighbors(cudaStream_t st, int64_t n, int64_t first, const double4 *x4,
                           const int32_t *cell_of, const int32_t *cell_start,
                           const int32_t *cell_list, int64_t cell_base, int3 dims,
                           double horizon, const int64_t *slice_ptr, int32_t *nbr) {
    if (n <= 0) return;
    k_neighbors<true><<<grid_for(n), kThreads, 0, st>>>(n, first, x4, cell_of, cell_start,
                                                        cell_list, cell_base, dims, horizon,
                                                        nullptr, slice_ptr, nbr); pd::note_launch();
}

void launch_cell_ids(cudaStream_t st, int64_t n, int64_t first, const double4 *x4, double3 lo, double cell,
                     int3 dims, int64_t cell_base, int32_t *cell_of, int32_t *count) {
    if (n <= 0) return;
    k_cell_ids<<<grid_for(n), kThreads, 0, st>>>(n, first, x4, lo, cell, dims, cell_base, cell_of, count);
    pd::note_launch();
}

void launch_cell_scatter(cudaStream_t st, int64_t n, int64_t first, const int32_t *cell_of, int32_t *cursor,
                         int32_t *cell_list) {
    if (n <= 0) return;
    k_cell_scatter<<<grid_for(n), kThreads, 0, st>>>(n, first, cell_of, cursor, cell_list);
    pd::note_launch();
}

void launch_sort_neighbors(cudaStream_t st, int64_t N, const int64_t *slice_ptr,
                           const int32_t *cnt, int32_t *nbr) {
    k_sort_neighbors<<<grid_for(N), kThreads, 0, st>>>(N, slice_ptr, cnt, nbr); pd::note_launch();
}

void launch_init_intact(cudaStream_t st, int64_t N, const int64_t *slice_ptr,
                        const int32_t *cnt, uint32_t *words) {
    k_init_intact<<<grid_for(N), kThreads, 0, st>>>(N, slice_ptr, cnt, words); pd::note_launch();
}

void launch_layout_union(cudaStream_t st, int64_t S, int64_t N, const int64_t *slice_ptr, const int32_t *cnt,
                         const int32_t *nbr_b, int32_t force_explicit, int64_t ustride, int32_t *mode, int32_t *len,
                         int32_t *uni) {
    if (S <= 0) return;
    const int64_t threads = S * 32;
    k_layout_union<<<(unsigned)((threads + kThreads - 1) / kThreads), kThreads, 0, st>>>(
        S, N, slice_ptr, cnt, nbr_b, force_explicit, ustride, mode, len, uni);
    pd::note_launch();
}

void launch_layout_fill(cudaStream_t st, int64_t N, const int64_t *slice_ptr, const int32_t *cnt,
                        const int32_t *nbr_b, const uint32_t *w_b, const SliceInfo *si, const int32_t *ulen,
                        int64_t ustride, const int32_t *uni, int32_t *nbr, uint32_t *words, uint32_t *fam,
                        int32_t *cnt_rt) {
    if (N <= 0) return;
    k_layout_fill<<<grid_for(N), kThreads, 0, st>>>(N, slice_ptr, cnt, nbr_b, w_b, si, ulen, ustride, uni, nbr,
                                                      words, fam, cnt_rt);
    pd::note_launch();
}

void launch_popcount(cudaStream_t st, int64_t N, const SliceInfo *si, const int32_t *cnt,
                     const uint32_t *words, int32_t *out) {
    k_popcount<<<grid_for(N), kThreads, 0, st>>>(N, si, cnt, words, out); pd::note_launch();
}

void launch_weighted_volume(cudaStream_t st, const Geo &g, double2 *mth) {
    k_weighted_volume<<<grid_for(g.N), kThreads, 0, st>>>(g, mth); pd::note_launch();
}

void launch_theta_serial(cudaStream_t st, const Geo &g, const double4 *y, const uint32_t *win,
                         double2 *mth, int64_t p0, int64_t p1) {
    if (p1 <= p0) return;
    k_theta_serial<<<grid_for(p1 - p0), kThreads, 0, st>>>(g, y, win, mth, p0, p1); pd::note_launch();
}

void launch_td_serial(cudaStream_t st, const Geo &g, const double4 *y, const double2 *mth,
                      const uint32_t *win, uint32_t *wout, int64_t p0, int64_t p1) {
    if (p1 <= p0) return;
    k_td_serial<<<grid_for(p1 - p0), kThreads, 0, st>>>(g, y, mth, win, wout, p0, p1);
    pd::note_launch();
}

void launch_force_serial(cudaStream_t st, const Geo &g, const double4 *y, const double2 *mth,
                         const uint32_t *win, uint32_t *wout, double4 *f, int accumulate,
                         int64_t p0, int64_t p1) {
    if (p1 <= p0) return;
    k_force_serial<<<grid_for(p1 - p0), kThreads, 0, st>>>(g, y, mth, win, wout, f, accumulate,
                                                           p0, p1); pd::note_launch();
}

void launch_kick_drift(cudaStream_t st, int64_t N, double c, double dt, const double4 *f,
                       double4 *v, double4 *y) {
    k_kick_drift<<<grid_for(N, 256), 256, 0, st>>>(N, c, dt, f, v, y); pd::note_launch();
}

void launch_kick(cudaStream_t st, int64_t N, double c, const double4 *f, double4 *v) {
    k_kick<<<grid_for(N, 256), 256, 0, st>>>(N, c, f, v); pd::note_launch();
}

void launch_bc_pos(cudaStream_t st, const BCDev &bc, double dt, int dir, int64_t ts, double4 *y) {
    if (bc.n <= 0 || bc.kind == PD_BC_CONTAINER) return;  // ContainerBC.jl:58-61 keeps y
    k_bc_pos<<<grid_for(bc.n, 256), 256, 0, st>>>(bc, dt, dir, ts, y); pd::note_launch();
}

void launch_bc_vel(cudaStream_t st, const BCDev &bc, int dir, const double4 *y, double4 *v) {
    if (bc.n <= 0 || (bc.kind == PD_BC_CONTAINER && !bc.has_limits)) return;
    k_bc_vel<<<grid_for(bc.n, 256), 256, 0, st>>>(bc, dir, y, v); pd::note_launch();
}

void launch_bc_scale(cudaStream_t st, const BCDev &bc, double dt, double4 *y) {
    if (bc.sn > 0) {
        k_bc_scale<<<grid_for(bc.sn, 256), 256, 0, st>>>(bc, dt, y);
        pd::note_launch();
    }
    launch_bc_snapshot(st, bc, y);
}

void launch_bc_snapshot(cudaStream_t st, const BCDev &bc, const double4 *y) {
    if (bc.n <= 0) return;
    k_bc_snapshot<<<grid_for(bc.n, 256), 256, 0, st>>>(bc, y); pd::note_launch();
}

void launch_momentum(cudaStream_t st, int64_t N, const double *mass, const double4 *v,
                     double4 *p) {
    k_momentum<<<grid_for(N, 256), 256, 0, st>>>(N, mass, v, p); pd::note_launch();
}

void launch_zero4(cudaStream_t st, int64_t N, double4 *a) {
    k_zero4<<<grid_for(N, 256), 256, 0, st>>>(N, a); pd::note_launch();
}

void launch_gate_multi(cudaStream_t st, const GateItem *items, int nitems, int gx, const double4 *x4,
                       const double4 *y, double *partials, int32_t *deformed) {
    if (nitems <= 0) return;
    k_gate_partial<<<dim3(gx, nitems), kGateThreads, 0, st>>>(items, gx, x4, y, partials, deformed);
    pd::note_launch();
    k_gate_final<<<(nitems + 127) / 128, 128, 0, st>>>(items, nitems, gx, partials, deformed);
    pd::note_launch();
}

void launch_damage(cudaStream_t st, int64_t N, const SliceInfo *si, const int32_t *cnt,
                   const uint32_t *words, const int32_t *intact0, const int32_t *tinfo,
                   double *damage) {
    k_damage<<<grid_for(N), kThreads, 0, st>>>(N, si, cnt, words, intact0, tinfo, damage); pd::note_launch();
}

void launch_sum4(cudaStream_t st, int64_t N, const double4 *a, double *partials, double *out3) {
    k_sum4_partial<<<kSumBlocks, 256, 0, st>>>(N, a, partials); pd::note_launch();
    k_sum4_final<<<1, 1, 0, st>>>(partials, out3); pd::note_launch();
}

void launch_unpack3(cudaStream_t st, int64_t n, const double *src3, const int64_t *map,
                    double4 *dst) {
    if (n <= 0) return;
    k_unpack3<<<grid_for(n, 256), 256, 0, st>>>(n, src3, map, dst); pd::note_launch();
}

void launch_pack3(cudaStream_t st, int64_t n, const double4 *src, const int64_t *map,
                  double *dst3) {
    if (n <= 0) return;
    k_pack3<<<grid_for(n, 256), 256, 0, st>>>(n, src, map, dst3); pd::note_launch();
}

void launch_nonfinite(cudaStream_t st, int64_t N, const double4 *a, int32_t *flag) {
    k_nonfinite<<<grid_for(N, 256), 256, 0, st>>>(N, a, flag); pd::note_launch();
}

}  // namespace pd
