// pd_internal.h -- device data layout and launcher declarations shared by
// the translation units of libperidyn_b200.so.
//
// Layout in HBM (one environment):
//  * Particles are stored in "internal" order: the environment order with
//    each material block padded to a multiple of 32 particles, so that a
//    32-particle slice never straddles two blocks.  Padding particles have
//    tinfo == -1 and no bonds.
//  * Per particle (array of structures, 32-byte aligned):
//      x4[i]  = (x0, x1, x2, volume)        reference configuration
//      y[i]   = (y0, y1, y2, -)             deformed position (FP64)
//      v[i], f[i], p[i]                     velocity, acceleration, momentum
//      mth[i] = (m, theta)                  weighted volume, dilatation
//      tinfo[i] = block << 8 | local type   (-1 for padding)
//  * Families are built in SELL-32 form ("build layout"): slice s holds
//    particles 32s..32s+31 and the k-th bond of lane l lives at
//    nbr[slice_ptr[s] + 32k + l].  Bonds of a particle are in descending
//    index order, the reference's family column order
//    (general_material.jl:88-90).
//  * The step kernels use the "runtime layout" (SliceInfo below): per slice
//    either one neighbour offset per slot shared by the 32 lanes (stencil)
//    or the build layout's explicit indices, plus intact and family-member
//    bit arrays with one 32-bit word per (lane, 32 slots).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/peridyn_b200.h"

namespace pd {

constexpr int kSlice = 32;
// Largest record staging plan of a slice (FP32C records of 32 bytes: 64 KB
// of shared memory per block).
constexpr int64_t kStageMaxRecords = 2048;

// Counts every kernel launch the library issues (pd_kernel_launches);
// graph replays add their kernel nodes.
void note_launch();
void add_launches(int64_t n);
int64_t launch_count();

struct DevBlock {
    int32_t kind;       // PD_MAT_*
    int32_t nt;         // types in the block
    int32_t pair_base;  // first PairParam of the block (nt*nt, column-major)
    int32_t type_base;  // first per-type density of the block
    int64_t first;      // first internal particle index (multiple of 32)
    int64_t n;          // particles (without padding)
    double c11;         // PMB bond stiffness bond_stiffness[1,1]
    float c11f;         // FP32 copy
    float pad0;
    double3 center;     // FP32C coordinate origin of the block
};

// Bond storage of one 32-particle slice (runtime layout).  Slot k of lane
// l is bond k of particle 32s + l; bit k%32 of word
// words[word + 32*(k/32) + l] is its intact flag (a second array of the same
// layout marks which slots hold a family member at all).
//  kExplicit: the neighbour is nbr[nbr + 32k + l] (int32, internal index).
//  kStencil:  every lane's slot k has the same index offset: the
//             neighbour is p + nbr[nbr + k].  Slots a particle does not use
//             are permanently 0 bits.  Warps then gather contiguous
//             neighbour records and no per-bond index is read at all.
// Slots are in descending offset order, so each particle meets its bonds in
// descending neighbour index -- the reference's family order.
constexpr int kExplicit = 0, kStencil = 1;
// Zero entries appended to the neighbour-index array (read-ahead margin of
// the stencil walks).
constexpr int64_t kNbrPad = 16;
struct SliceInfo {
    int64_t nbr;   // offset into nbr[]
    int64_t word;  // offset into the bit arrays
    int32_t len;   // slots per particle, multiple of 32
    int32_t mode;  // kExplicit / kStencil
};

// Access to one particle's bonds.
struct BondRef {
    const int32_t *nb;
    uint32_t *w;
    int32_t mode;
    int32_t p;
    __device__ __forceinline__ int32_t q(int32_t k) const { return mode == kStencil ? p + nb[k] : nb[32 * k]; }
    __device__ __forceinline__ uint32_t *word(int32_t k) const { return w + 32 * (k >> 5); }
};

__device__ __forceinline__ BondRef bond_ref(const SliceInfo *si, const int32_t *nbr, const uint32_t *words,
                                            int64_t p) {
    const SliceInfo s = si[p >> 5];
    BondRef b;
    b.mode = s.mode;
    b.p = (int32_t)p;
    b.nb = nbr + s.nbr + (s.mode == kStencil ? 0 : (p & 31));
    b.w = const_cast<uint32_t *>(words) + s.word + (p & 31);
    return b;
}

struct PairParam {
    double cs;    // critical stretch
    double k35;   // 3K - 5G (LPS); 3K (elasto-plastic)
    double g15;   // 15G
    double psi2;  // 2 psi (elasto-plastic yield value)
};

// Everything a bond kernel reads (passed by value).
struct Geo {
    int64_t N;                 // internal particle count (multiple of 32)
    const double4 *x4;         // (x, vol)
    const int32_t *tinfo;
    const DevBlock *blocks;
    const PairParam *pairs;
    const double *tdens;       // per block-type density
    const SliceInfo *si;       // N/32 slice descriptors
    const int32_t *cnt;        // slots to scan per particle
    const int32_t *nbr;        // bond index data (see SliceInfo)
    const uint32_t *fam;       // family-member bits (same layout as intact)
    const int32_t *deformed;   // per block
    // elasto-plastic blocks: td_norm2 per particle, plastic deviatoric
    // strain per bond slot (read from edp_in, written to edp_out)
    double *td2;
    const double *edp_in;
    double *edp_out;
};

// Per-slot double index of bond slot k of particle p (elasto-plastic edp).
__device__ __forceinline__ int64_t slot_index(const SliceInfo *si, int64_t p, int32_t k) {
    return ((si[p >> 5].word + 32 * (int64_t)(k >> 5) + (p & 31)) << 5) + (k & 31);
}

// Slot of neighbour p in q's family: slots hold descending neighbour
// indices (stencil slices: descending offsets), so a binary search.
__device__ __forceinline__ int32_t slot_of(const SliceInfo *si, const int32_t *nbr, const int32_t *cnt, int64_t q,
                                           int64_t p) {
    const SliceInfo s = si[q >> 5];
    const bool st = s.mode == kStencil;
    const int32_t *nb = nbr + s.nbr + (st ? 0 : (q & 31));
    const int32_t target = st ? (int32_t)(p - q) : (int32_t)p;
    int32_t lo = 0, hi = cnt[q];
    while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        const int32_t v = st ? nb[mid] : nb[32 * mid];
        if (v > target) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

struct BCDev {
    int32_t kind;
    int32_t dims;      // bit d set: dimension d constrained
    double rate[3];
    double scale[3], fix[3];  // DeltaScale / ScaleFixWait
    double lo[3], hi[3];      // Container limits
    int32_t has_limits, pad;
    int64_t n;
    const int32_t *idx;  // internal indices, ascending
    double4 *last;       // BC.last per constrained particle
    int64_t sn;          // ScaleFixWait: particles scaled at check time
    const int32_t *sidx;
};

// ---------------------------------------------------------------------
// Launchers (pd_exact.cu, compiled with -fmad=false)
// ---------------------------------------------------------------------
// Family build.
// Cell binning of one block: cell ids (into the concatenated grids) and
// per-cell counts, then, from the cell starts, the cell lists.
void launch_cell_ids(cudaStream_t st, int64_t n, int64_t first, const double4 *x4, double3 lo, double cell,
                     int3 dims, int64_t cell_base, int32_t *cell_of, int32_t *count);
void launch_cell_scatter(cudaStream_t st, int64_t n, int64_t first, const int32_t *cell_of, int32_t *cursor,
                         int32_t *cell_list);
void launch_count_neighbors(cudaStream_t st, int64_t n, int64_t first, const double4 *x4,
                            const int32_t *cell_of, const int32_t *cell_start,
                            const int32_t *cell_list, int64_t cell_base, int3 dims,
                            double horizon, int32_t *cnt);
void launch_fill_neighbors(cudaStream_t st, int64_t n, int64_t first, const double4 *x4,
                           const int32_t *cell_of, const int32_t *cell_start,
                           const int32_t *cell_list, int64_t cell_base, int3 dims,
                           double horizon, const int64_t *slice_ptr, int32_t *nbr);
void launch_sort_neighbors(cudaStream_t st, int64_t N, const int64_t *slice_ptr,
                           const int32_t *cnt, int32_t *nbr);
void launch_init_intact(cudaStream_t st, int64_t N, const int64_t *slice_ptr,
                        const int32_t *cnt, uint32_t *words);
// Runtime layout built on the device from the build layout: per-slice
// unions and stencil decision (mode, len, union offsets at s * ustride),
// then the runtime arrays (nbr, words, fam zeroed beforehand; cnt_rt).
void launch_layout_union(cudaStream_t st, int64_t S, int64_t N, const int64_t *slice_ptr, const int32_t *cnt,
                         const int32_t *nbr_b, int32_t force_explicit, int64_t ustride, int32_t *mode, int32_t *len,
                         int32_t *uni);
void launch_layout_fill(cudaStream_t st, int64_t N, const int64_t *slice_ptr, const int32_t *cnt,
                        const int32_t *nbr_b, const uint32_t *w_b, const SliceInfo *si, const int32_t *ulen,
                        int64_t ustride, const int32_t *uni, int32_t *nbr, uint32_t *words, uint32_t *fam,
                        int32_t *cnt_rt);
// Runtime layout (SliceInfo) from here on.
void launch_popcount(cudaStream_t st, int64_t N, const SliceInfo *si, const int32_t *cnt,
                     const uint32_t *words, int32_t *out);
void launch_weighted_volume(cudaStream_t st, const Geo &g, double2 *mth);

// Serial-order FP64 force path.
void launch_theta_serial(cudaStream_t st, const Geo &g, const double4 *y, const uint32_t *win,
                         double2 *mth, int64_t p0, int64_t p1);
void launch_force_serial(cudaStream_t st, const Geo &g, const double4 *y, const double2 *mth,
                         const uint32_t *win, uint32_t *wout, double4 *f, int accumulate,
                         int64_t p0, int64_t p1);
// elasto_plastic.jl:166-172 out_of_loop! td_norm2 pass (breaks bonds too)
void launch_td_serial(cudaStream_t st, const Geo &g, const double4 *y, const double2 *mth,
                      const uint32_t *win, uint32_t *wout, int64_t p0, int64_t p1);

// Elementwise velocity-Verlet pieces (exact FP64 arithmetic).
void launch_kick_drift(cudaStream_t st, int64_t N, double c, double dt, const double4 *f,
                       double4 *v, double4 *y);
void launch_kick(cudaStream_t st, int64_t N, double c, const double4 *f, double4 *v);
// ts: time_step when the position BC is applied (DeltaScale)
void launch_bc_pos(cudaStream_t st, const BCDev &bc, double dt, int dir, int64_t ts, double4 *y);
// y: positions at the velocity BC (Container)
void launch_bc_vel(cudaStream_t st, const BCDev &bc, int dir, const double4 *y, double4 *v);
void launch_bc_snapshot(cudaStream_t st, const BCDev &bc, const double4 *y);
// ScaleFixWait check!: scale the scalebool particles, then re-read last.
void launch_bc_scale(cudaStream_t st, const BCDev &bc, double dt, double4 *y);
void launch_momentum(cudaStream_t st, int64_t N, const double *mass, const double4 *v,
                     double4 *p);
void launch_zero4(cudaStream_t st, int64_t N, double4 *a);

// Deformed gate (general_material.jl:243-255), for every listed block in
// two launches: grid.y = list entry, grid.x = gx CTAs per block.
struct GateItem {
    int64_t first, n;
    int32_t block, pad;
};
void launch_gate_multi(cudaStream_t st, const GateItem *items, int nitems, int gx, const double4 *x4,
                       const double4 *y, double *partials, int32_t *deformed);

// Damage / diagnostics.
void launch_damage(cudaStream_t st, int64_t N, const SliceInfo *si, const int32_t *cnt,
                   const uint32_t *words, const int32_t *intact0, const int32_t *tinfo,
                   double *damage);
void launch_sum4(cudaStream_t st, int64_t N, const double4 *a, double *partials, double *out3);

// Layout conversion between the reference's 3xN column-major arrays and
// internal double4 arrays.  map[e] = internal index of environment index e.
void launch_unpack3(cudaStream_t st, int64_t n, const double *src3, const int64_t *map,
                    double4 *dst);
void launch_pack3(cudaStream_t st, int64_t n, const double4 *src, const int64_t *map,
                  double *dst3);
void launch_nonfinite(cudaStream_t st, int64_t N, const double4 *a, int32_t *flag);

}  // namespace pd
