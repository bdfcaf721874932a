// Fused docking kernels (sm_100a).  One rotation's score grid is produced by
// three plane/line passes that never store the full forward spectrum of the
// ligand nor the full score grid:
//
//   K1 plane_fwd   (rotation, voxel x-plane p): rotate the ligand, voxelize
//                  plane p (rPSC real part + charge imaginary part, bit-exact
//                  with MEGADOCK's CPU path), 2D forward FFT over (y, z) in
//                  shared memory, store the plane's spectrum  A[p][ky][kz].
//   K2 xline       (rotation, ky, 32 kz lines): forward FFT along x of the
//                  ng non-zero planes, multiply by conj(R^), inverse FFT along
//                  x, store G[x][ky][kz].
//   K3 plane_inv   (rotation, x-plane): inverse FFT over (ky, kz) -> real score
//                  plane, per-plane top-t candidates.
//   K4 merge       (rotation): top-t of the per-plane candidates with
//                  MEGADOCK's selection rules -> pose records.
//
// References (MEGADOCK, akiyamalab):
//   rotation           src/docking.cpp:368-396
//   rPSC voxelization  src/ligand.cpp:20-198 (+ precalc :241-260, voxel_init
//                      src/protein.cpp:134-165)
//   charges            src/ligand.cpp:200-239
//   embedding          src/fft_process.cpp:306-330
//   FFT / product      src/fft_process.cpp:333-396 (FFTW) and :537-558 (cuFFT)
//   top-t              src/fft_process.cpp:399-458
#pragma once
#include <climits>

#include "fft_dev.cuh"

namespace mdb {

constexpr int kNT = 512;          // threads per CTA for the plane kernels
#ifndef MDB_K1_NT
#define MDB_K1_NT 1024
#endif
constexpr int kNT1 = MDB_K1_NT;   // threads per CTA of the forward plane kernel (one CTA per SM)
constexpr int kLT = 32;           // lines per CTA in the x-line kernel
constexpr int kMaxLigAtoms = 32768;

struct DevPose {
    float score;
    int rot, i, j, k;
};

struct LigandView {
    int na;
    const float4 *__restrict__ atom;   // centred x, y, z and charge
    const float2 *__restrict__ rad2;   // (R^2 * 1.5, R^2 * 1.0)
    float delta;                       // ligand core value (-b)
};

struct GridView {
    int ng;                            // voxel edge (N/2)
    float gw;                          // grid width (Protein::grid_width)
    float pad;                         // ng * gw / 2 (Ligand::electro)
    const float *__restrict__ gc;      // grid centre coordinates [ng]
    const float2 *__restrict__ tw;     // exp(-2 pi i j / N), j < N
};

// ------------------------------------------------------------------ voxelization
// Shared-memory bit planes for one CTA's x-plane p.
template <int NG>
struct VoxShared {
    static constexpr int W = (NG + 31) / 32;
    uint32_t core[5][NG * W];   // planes p-2 .. p+2
    uint32_t surf[3][NG * W];   // planes p-1 .. p+1
};

__device__ __forceinline__ float rot_x(const float *m, float x, float y, float z) {
    // (m0*x + m1*y) + m2*z in float, no contraction (src/docking.cpp:390-392)
    return __fadd_rn(__fadd_rn(__fmul_rn(m[0], x), __fmul_rn(m[1], y)), __fmul_rn(m[2], z));
}

// (int)(c / gw + ng/2), the atom's nearest-cell search origin (src/ligand.cpp:71-73)
__device__ __forceinline__ int box_origin(float c, float gw, int ng) {
    return __float2int_rz(__fadd_rn(__fdiv_rn(c, gw), (float)(ng / 2)));
}

// clamp((int)((c + pad) / gw)), the charge cell (src/ligand.cpp:219-221)
__device__ __forceinline__ int charge_cell(float c, float pad, float gw, int ng) {
    int v = __float2int_rz(__fdiv_rn(__fadd_rn(c, pad), gw));
    return max(0, min(ng - 1, v));
}

__device__ __forceinline__ float sqdist(float c, float g) {
    const float d = __fsub_rn(c, g);
    return __fmul_rn(d, d);
}

template <int NG>
__device__ __forceinline__ bool vbit(const uint32_t *plane, int q, int s) {
    constexpr int W = VoxShared<NG>::W;
    return (plane[q * W + (s >> 5)] >> (s & 31)) & 1u;
}

// Per-rotation atom record for the voxelizer: rotated coordinates, the
// search-box origin (src/ligand.cpp:71-73) and both sphere radii squared.
struct MarkEntry {
    float4 pos;   // rotated x, y, z and R^2 * 1.5
    int4 box;     // search-box origin i, j, k and R^2 * 1.0 (as bits)
};

// Shape buckets: atoms are grouped by box origin i, shifted by kReach so that
// origins in [-kReach, ng + kReach) map to [0, ng + 2 kReach).
constexpr int kReach = 4;

// Mark core / surface bits of the planes around p.  The atoms whose box can
// reach those planes are the contiguous bucket range [lo, hi) of the rotation's
// record array; every (atom, plane, row) of their boxes is one task, spread
// evenly over the block; a task tests the row's cells and ORs the bits (the
// marks are ORs, so the order of atoms does not matter).
template <int NG>
__device__ void vox_mark(VoxShared<NG> &vs, const MarkEntry *__restrict__ rec, int lo, int hi, const GridView &G,
                         int p, bool general_delta) {
    constexpr int W = VoxShared<NG>::W;
    const int ng = G.ng;
    const int plo = general_delta ? -2 : -1;
    const int nplanes = general_delta ? 5 : 3;
    const int ntask = (hi - lo) * nplanes * 5;
    for (int task = threadIdx.x; task < ntask; task += blockDim.x) {
        const int e = task / (nplanes * 5);
        const int rem = task % (nplanes * 5);
        const int i = p + plo + rem / 5;
        const MarkEntry me = rec[lo + e];
        const int j = me.box.y - 2 + rem % 5;
        if (i < 0 || i >= ng || i < me.box.x - 2 || i > me.box.x + 2 || j < 0 || j >= ng) continue;
        const float rc2 = me.pos.w, rs2 = __int_as_float(me.box.w);
        const float d2 = __fadd_rn(sqdist(me.pos.x, __ldg(&G.gc[i])), sqdist(me.pos.y, __ldg(&G.gc[j])));
        // d3 = d2 + dz^2 >= d2 and R^2 <= 1.5 R^2: a row outside the core
        // disc has no cell in either sphere
        if (!(d2 < rc2)) continue;
        // the row's (at most 5) cells as bits of a 64-bit window from word wb
        const int ka = max(me.box.z - 2, 0), kb = min(me.box.z + 3, ng);
        const int wb = ka >> 5;
        unsigned long long cm = 0ull, sm = 0ull;
        for (int k = ka; k < kb; ++k) {
            const float d3 = __fadd_rn(d2, sqdist(me.pos.z, __ldg(&G.gc[k])));
            const unsigned long long bit = 1ull << (k - 32 * wb);
            if (d3 < rc2) cm |= bit;
            if (d3 < rs2) sm |= bit;
        }
        const int slot = i - p + 2;
        const bool do_surf = (i >= p - 1 && i <= p + 1);
        uint32_t *crow = &vs.core[slot][j * W + wb];
        if ((uint32_t)cm) atomicOr(crow, (uint32_t)cm);
        if (cm >> 32) atomicOr(crow + 1, (uint32_t)(cm >> 32));
        if (do_surf) {
            uint32_t *srow = &vs.surf[slot - 1][j * W + wb];
            if ((uint32_t)sm) atomicOr(srow, (uint32_t)sm);
            if (sm >> 32) atomicOr(srow + 1, (uint32_t)(sm >> 32));
        }
    }
    __syncthreads();
}

// Word-parallel form of vox_code: the class bits of 32 cells (row q, word w)
// of plane p at once.  c2 = "value delta", c1 = "value 1.0".
template <int NG>
__device__ __forceinline__ uint32_t vw_core(const VoxShared<NG> &vs, int slot, int q, int w) {
    constexpr int W = VoxShared<NG>::W;
    return (q < 0 || q >= NG || w < 0 || w >= W) ? 0u : vs.core[slot][q * W + w];
}

template <int NG>
__device__ __forceinline__ uint32_t vw_surf(const VoxShared<NG> &vs, int slot, int q, int w) {
    constexpr int W = VoxShared<NG>::W;
    return (q < 0 || q >= NG || w < 0 || w >= W) ? 0u : vs.surf[slot - 1][q * W + w];
}

// bits s of word w with 1 <= s <= ng - 2
__device__ __forceinline__ uint32_t vw_inner(int w, int ng) {
    uint32_t m = 0xffffffffu;
    const int s0 = 32 * w;
    if (s0 < 1) m &= ~1u;
    const int hi = ng - 2 - s0;   // last kept bit
    if (hi < 0) return 0u;
    if (hi < 31) m &= (2u << hi) - 1u;
    return m;
}

// core cells of (slot, q, w) that survive the scrape (vox_surv)
template <int NG>
__device__ __forceinline__ uint32_t vw_surv(const VoxShared<NG> &vs, int slot, int i, int q, int w, int ng) {
    const uint32_t c = vw_core<NG>(vs, slot, q, w);
    if (!c) return 0u;
    const uint32_t left = (c << 1) | (vw_core<NG>(vs, slot, q, w - 1) >> 31);    // core at s - 1
    const uint32_t right = (c >> 1) | (vw_core<NG>(vs, slot, q, w + 1) << 31);   // core at s + 1
    const uint32_t nb = vw_core<NG>(vs, slot - 1, q, w) & vw_core<NG>(vs, slot + 1, q, w) &
                        vw_core<NG>(vs, slot, q - 1, w) & vw_core<NG>(vs, slot, q + 1, w) & left & right;
    const bool inner_iq = i >= 1 && i <= ng - 2 && q >= 1 && q <= ng - 2;
    const uint32_t interior = inner_iq ? vw_inner(w, ng) : 0u;
    return c & (~interior | nb);
}

// cells of class 0 (neither a surviving core cell nor a surface cell)
template <int NG>
__device__ __forceinline__ uint32_t vw_empty(const VoxShared<NG> &vs, int slot, int i, int q, int w, int ng) {
    return ~(vw_surv<NG>(vs, slot, i, q, w, ng) | vw_surf<NG>(vs, slot, q, w));
}

template <int NG>
__device__ __forceinline__ void vox_code_words(const VoxShared<NG> &vs, int p, int q, int w, int ng,
                                               bool general_delta, uint32_t &c2, uint32_t &c1) {
    const uint32_t surv = vw_surv<NG>(vs, 2, p, q, w, ng);
    c2 = surv;
    c1 = vw_surf<NG>(vs, 2, q, w) & ~surv;
    if (!general_delta || !surv) return;
    if (!(p >= 1 && p <= ng - 2 && q >= 1 && q <= ng - 2)) return;
    const uint32_t e0 = vw_empty<NG>(vs, 2, p, q, w, ng);
    const uint32_t es = (e0 << 1) | (vw_empty<NG>(vs, 2, p, q, w - 1, ng) >> 31) | (e0 >> 1) |
                        (vw_empty<NG>(vs, 2, p, q, w + 1, ng) << 31);
    const uint32_t ez = vw_empty<NG>(vs, 1, p - 1, q, w, ng) | vw_empty<NG>(vs, 3, p + 1, q, w, ng) |
                        vw_empty<NG>(vs, 2, p, q - 1, w, ng) | vw_empty<NG>(vs, 2, p, q + 1, w, ng);
    const uint32_t demote = surv & vw_inner(w, ng) & (es | ez);
    c2 = surv & ~demote;
    c1 |= demote;
}

// Core bit survives the swollen-surface scrape (src/ligand.cpp:110-134):
// interior cells with a 6-neighbour outside the core lose their core value.
template <int NG>
__device__ __forceinline__ bool vox_surv(const VoxShared<NG> &vs, int slot, int i, int q, int s, int ng) {
    const uint32_t *c = vs.core[slot];
    if (!vbit<NG>(c, q, s)) return false;
    const bool interior = i >= 1 && i <= ng - 2 && q >= 1 && q <= ng - 2 && s >= 1 && s <= ng - 2;
    if (!interior) return true;
    return vbit<NG>(vs.core[slot - 1], q, s) && vbit<NG>(vs.core[slot + 1], q, s) && vbit<NG>(c, q - 1, s) &&
           vbit<NG>(c, q + 1, s) && vbit<NG>(c, q, s - 1) && vbit<NG>(c, q, s + 1);
}

// Pre-step-4 value class: 2 = core (delta), 1 = surface (1.0), 0 = empty.
template <int NG>
__device__ __forceinline__ int vox_class(const VoxShared<NG> &vs, int slot, int i, int q, int s, int ng) {
    if (vox_surv<NG>(vs, slot, i, q, s, ng)) return 2;
    return vbit<NG>(vs.surf[slot - 1], q, s) ? 1 : 0;
}

// Real rPSC class of cell (p, q, s): 2 = core (value delta), 1 = surface
// (value 1.0), 0 = empty.  With delta != 1 the interior core cells next to an
// empty cell become surface (src/ligand.cpp:176-195).
template <int NG>
__device__ __forceinline__ int vox_code(const VoxShared<NG> &vs, int p, int q, int s, int ng, bool general_delta) {
    const int c = vox_class<NG>(vs, 2, p, q, s, ng);
    if (c != 2 || !general_delta) return c;
    const bool interior = p >= 1 && p <= ng - 2 && q >= 1 && q <= ng - 2 && s >= 1 && s <= ng - 2;
    if (interior) {
        if (vox_class<NG>(vs, 1, p - 1, q, s, ng) == 0 || vox_class<NG>(vs, 3, p + 1, q, s, ng) == 0 ||
            vox_class<NG>(vs, 2, p, q - 1, s, ng) == 0 || vox_class<NG>(vs, 2, p, q + 1, s, ng) == 0 ||
            vox_class<NG>(vs, 2, p, q, s - 1, ng) == 0 || vox_class<NG>(vs, 2, p, q, s + 1, ng) == 0)
            return 1;
    }
    return 2;
}

// ------------------------------------------------------------------ atom prep
// Once per rotation: rotate every atom (src/docking.cpp:386-393), compute its
// search-box origin and its charge cell (src/ligand.cpp:71-73, 219-221) and
// bucket the atoms by x-plane:
//  * shape records rec[b][.] grouped by box origin i (any order inside a
//    bucket), bucket starts sstart[b][0 .. ng + 2 kReach];
//  * charge entries cq[b][.] = (cell j * ng + k, charge bits) grouped by the
//    charge cell's plane, in ascending atom order inside a bucket (the order
//    in which MEGADOCK adds charges), bucket starts cstart[b][0 .. ng].
constexpr int kNTP = 256;

template <int NG>
__global__ void __launch_bounds__(kNTP)
    k_atom_prep(LigandView L, GridView G, const float *__restrict__ rotm, MarkEntry *__restrict__ rec,
                int *__restrict__ sstart, int2 *__restrict__ cq, int *__restrict__ cstart) {
    constexpr int NBS = NG + 2 * kReach;
    __shared__ int cnt_s[NBS], cnt_c[NG], cur_s[NBS], cur_c[NG];
    __shared__ float m[9];
    const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31;
    if (tid < 9) m[tid] = rotm[(size_t)b * 9 + tid];
    for (int i = tid; i < NBS; i += blockDim.x) cnt_s[i] = 0;
    for (int i = tid; i < NG; i += blockDim.x) cnt_c[i] = 0;
    __syncthreads();
    for (int l = tid; l < L.na; l += blockDim.x) {
        const float4 a = __ldg(&L.atom[l]);
        const float xr = rot_x(m, a.x, a.y, a.z);
        const int sb = box_origin(xr, G.gw, G.ng) + kReach;
        if (sb >= 0 && sb < NBS) atomicAdd(&cnt_s[sb], 1);
        atomicAdd(&cnt_c[charge_cell(xr, G.pad, G.gw, G.ng)], 1);
    }
    __syncthreads();
    int *ss = sstart + (size_t)b * (NBS + 1);
    int *cs = cstart + (size_t)b * (NG + 1);
    if (tid == 0) {
        int acc = 0;
        for (int i = 0; i < NBS; ++i) {
            ss[i] = acc;
            cur_s[i] = acc;
            acc += cnt_s[i];
        }
        ss[NBS] = acc;
        acc = 0;
        for (int i = 0; i < NG; ++i) {
            cs[i] = acc;
            cur_c[i] = acc;
            acc += cnt_c[i];
        }
        cs[NG] = acc;
    }
    __syncthreads();
    MarkEntry *rb = rec + (size_t)b * L.na;
    for (int l = tid; l < L.na; l += blockDim.x) {
        const float4 a = __ldg(&L.atom[l]);
        const float xr = rot_x(m, a.x, a.y, a.z);
        const int i2 = box_origin(xr, G.gw, G.ng);
        const int sb = i2 + kReach;
        if (sb < 0 || sb >= NBS) continue;
        const float yr = rot_x(m + 3, a.x, a.y, a.z);
        const float zr = rot_x(m + 6, a.x, a.y, a.z);
        const float2 r2 = __ldg(&L.rad2[l]);
        const int pos = atomicAdd(&cur_s[sb], 1);
        rb[pos].pos = make_float4(xr, yr, zr, r2.x);
        rb[pos].box = make_int4(i2, box_origin(yr, G.gw, G.ng), box_origin(zr, G.gw, G.ng), __float_as_int(r2.y));
    }
    // charge entries in atom order: warp 0 walks the atoms 32 at a time
    if (tid < 32) {
        int2 *qb = cq + (size_t)b * L.na;
        for (int base = 0; base < L.na; base += 32) {
            const int l = base + lane;
            int ie = -1, key = 0;
            float q = 0.f;
            if (l < L.na) {
                const float4 a = __ldg(&L.atom[l]);
                ie = charge_cell(rot_x(m, a.x, a.y, a.z), G.pad, G.gw, G.ng);
                const int je = charge_cell(rot_x(m + 3, a.x, a.y, a.z), G.pad, G.gw, G.ng);
                const int ke = charge_cell(rot_x(m + 6, a.x, a.y, a.z), G.pad, G.gw, G.ng);
                key = je * G.ng + ke;
                q = a.w;
            }
            const uint32_t grp = __match_any_sync(0xffffffffu, ie);
            int pos = 0;
            if (ie >= 0) pos = cur_c[ie] + __popc(grp & ((1u << lane) - 1u));
            __syncwarp();
            if (ie >= 0) {
                qb[pos] = make_int2(key, __float_as_int(q));
                if (lane == 31 - __clz(grp)) cur_c[ie] += __popc(grp);
            }
            __syncwarp();
        }
    }
}

// ------------------------------------------------------------------ K0
// Ligand grid of one (rotation, x-plane p), everything but the FFT:
//  * real part: core / surface marks of the atoms near p (task-parallel), the
//    swollen-surface scrape and the surface fill (src/ligand.cpp:20-198),
//    stored as two bit planes: vbits[b][p][0] = "value delta",
//    vbits[b][p][1] = "value 1.0";
//  * imaginary part: per-cell charge sums in ascending atom order from 0.0
//    (src/ligand.cpp:200-239), stored as a compact list of the plane's charged
//    cells qlist[b][p][e] = (q * NG + s, sum as bits), qcount[b][p] entries.
constexpr int kNT0 = 256;

// K0m: the core and surface marks of one (rotation, x-plane i), computed once
// per plane and stored for the K0 CTAs of planes i-2 .. i+2 (each of which
// would otherwise mark its neighbour planes itself):
//   marks[b][i][0] = core bits, marks[b][i][1] = surface bits (rows of W words).
// Same tests and rounding as vox_mark, so the bits are the same.
template <int NG>
__global__ void __launch_bounds__(kNT0)
    k_vox_mark(LigandView L, GridView G, const MarkEntry *__restrict__ rec, const int *__restrict__ sstart,
               uint32_t *__restrict__ marks) {
    constexpr int W = VoxShared<NG>::W;
    constexpr int NBS = NG + 2 * kReach;
    __shared__ uint32_t cs[2][NG * W];
    const int i = blockIdx.x, b = blockIdx.y, tid = threadIdx.x;
    for (int w = tid; w < 2 * NG * W; w += blockDim.x) (&cs[0][0])[w] = 0u;
    __syncthreads();
    const int ng = G.ng;
    const int *ss = sstart + (size_t)b * (NBS + 1);
    const int lo = ss[max(i - 2 + kReach, 0)], hi = ss[min(i + 2 + kReach + 1, NBS)];
    const MarkEntry *rb = rec + (size_t)b * L.na;
    for (int task = tid; task < (hi - lo) * 5; task += blockDim.x) {
        const MarkEntry me = rb[lo + task / 5];
        const int j = me.box.y - 2 + task % 5;
        if (i >= ng || i < me.box.x - 2 || i > me.box.x + 2 || j < 0 || j >= ng) continue;
        const float rc2 = me.pos.w, rs2 = __int_as_float(me.box.w);
        const float d2 = __fadd_rn(sqdist(me.pos.x, __ldg(&G.gc[i])), sqdist(me.pos.y, __ldg(&G.gc[j])));
        if (!(d2 < rc2)) continue;
        const int ka = max(me.box.z - 2, 0), kb = min(me.box.z + 3, ng);
        const int wb = ka >> 5;
        unsigned long long cm = 0ull, sm = 0ull;
        for (int k = ka; k < kb; ++k) {
            const float d3 = __fadd_rn(d2, sqdist(me.pos.z, __ldg(&G.gc[k])));
            const unsigned long long bit = 1ull << (k - 32 * wb);
            if (d3 < rc2) cm |= bit;
            if (d3 < rs2) sm |= bit;
        }
        uint32_t *crow = &cs[0][j * W + wb], *srow = &cs[1][j * W + wb];
        if ((uint32_t)cm) atomicOr(crow, (uint32_t)cm);
        if (cm >> 32) atomicOr(crow + 1, (uint32_t)(cm >> 32));
        if ((uint32_t)sm) atomicOr(srow, (uint32_t)sm);
        if (sm >> 32) atomicOr(srow + 1, (uint32_t)(sm >> 32));
    }
    __syncthreads();
    uint32_t *dst = marks + ((size_t)b * NG + i) * 2 * NG * W;
    for (int w = tid; w < 2 * NG * W; w += blockDim.x) dst[w] = (&cs[0][0])[w];
}

// Whether k_vox_bits keeps its bit planes (VoxShared) and output words in
// dynamic shared memory: where their static form would pass 40 KB of the 48 KB
// a kernel may declare statically (NG > 160).
template <int NG>
constexpr bool vox_bits_dyn() {
    return sizeof(VoxShared<NG>) + sizeof(uint32_t) * 2 * NG * VoxShared<NG>::W > 40 * 1024;
}

// Whether k_vox_bits keeps the first charge entry of each cell in shared
// memory (an int per cell): where it fits beside the dynamic bit planes in a
// CTA's 227 KB (ng1 <= 200).  Above, each entry finds out whether it is its
// cell's first by scanning the plane's earlier entries (a plane holds the
// charges of a few hundred atoms at most).
template <int NG>
constexpr bool vox_first_smem() {
    return sizeof(int) * NG * NG +
               (vox_bits_dyn<NG>() ? sizeof(VoxShared<NG>) + sizeof(uint32_t) * 2 * NG * VoxShared<NG>::W : 0) <=
           226 * 1024;   // a KB left for the kernel's static shared memory
}

// Dynamic shared memory of k_vox_bits: the first charge entry of each cell
// (vox_first_smem), then (vox_bits_dyn) the bit planes and the output words.
template <int NG>
constexpr size_t vox_bits_smem() {
    return (vox_first_smem<NG>() ? sizeof(int) * NG * NG : 0) +
           (vox_bits_dyn<NG>() ? sizeof(VoxShared<NG>) + sizeof(uint32_t) * 2 * NG * VoxShared<NG>::W : 0);
}

// PREMARKED: the marks come from K0m (marks != nullptr) instead of vox_mark.
template <int NG, bool PREMARKED = false>
__global__ void __launch_bounds__(kNT0)
    k_vox_bits(LigandView L, GridView G, const MarkEntry *__restrict__ rec, const int *__restrict__ sstart,
               const int2 *__restrict__ cq, const int *__restrict__ cstart, uint32_t *__restrict__ vbits,
               int2 *__restrict__ qlist, int *__restrict__ qcount, const uint32_t *__restrict__ marks = nullptr) {
    constexpr int W = VoxShared<NG>::W;
    constexpr int NBS = NG + 2 * kReach;
    __shared__ int count;
    constexpr bool FIRST = vox_first_smem<NG>();
    extern __shared__ __align__(16) int first[];   // NG * NG where FIRST (vox_bits_smem)
    VoxShared<NG> *vsp;
    uint32_t(*ob)[NG * W];
    if constexpr (vox_bits_dyn<NG>()) {
        vsp = reinterpret_cast<VoxShared<NG> *>(first + (FIRST ? NG * NG : 0));
        ob = reinterpret_cast<uint32_t(*)[NG * W]>(vsp + 1);
    } else {
        __shared__ VoxShared<NG> vs_static;
        __shared__ uint32_t ob_static[2][NG * W];
        vsp = &vs_static;
        ob = ob_static;
    }
    VoxShared<NG> &vs = *vsp;
    const int p = blockIdx.x, b = blockIdx.y, tid = threadIdx.x;
    const bool gd = (L.delta != 1.0f);
    if constexpr (PREMARKED) {
        // core of planes p-2 .. p+2 (p-1 .. p+1 unless delta != 1, as vox_mark
        // marks them), surface of p-1 .. p+1; planes outside the grid are 0
        const uint32_t *mb = marks + (size_t)b * NG * 2 * NG * W;
        for (int w = tid; w < 5 * NG * W; w += blockDim.x) {
            const int slot = w / (NG * W), i = p - 2 + slot;
            const bool on = (i >= 0 && i < G.ng && i < NG) && (gd || (slot >= 1 && slot <= 3));
            (&vs.core[0][0])[w] = on ? mb[(size_t)i * 2 * NG * W + w % (NG * W)] : 0u;
        }
        for (int w = tid; w < 3 * NG * W; w += blockDim.x) {
            const int i = p - 1 + w / (NG * W);
            const bool on = (i >= 0 && i < G.ng && i < NG);
            (&vs.surf[0][0])[w] = on ? mb[(size_t)i * 2 * NG * W + NG * W + w % (NG * W)] : 0u;
        }
    } else {
        for (int w = tid; w < 5 * NG * W; w += blockDim.x) (&vs.core[0][0])[w] = 0u;
        for (int w = tid; w < 3 * NG * W; w += blockDim.x) (&vs.surf[0][0])[w] = 0u;
    }
    for (int w = tid; w < 2 * NG * W; w += blockDim.x) (&ob[0][0])[w] = 0u;
    if constexpr (FIRST)
        for (int c = tid; c < NG * NG; c += blockDim.x) first[c] = 0x7fffffff;
    if (tid == 0) count = 0;
    __syncthreads();
    if constexpr (!PREMARKED) {
        const int reach = gd ? 4 : 3;
        const int *ss = sstart + (size_t)b * (NBS + 1);
        const int lo = ss[max(p - reach + kReach, 0)], hi = ss[min(p + reach + kReach + 1, NBS)];
        vox_mark<NG>(vs, rec + (size_t)b * L.na, lo, hi, G, p, gd);
    }
    for (int c = tid; c < NG * W; c += blockDim.x) {
        const int q = c / W, w = c % W;
        uint32_t c2, c1;
        vox_code_words<NG>(vs, p, q, w, NG, gd, c2, c1);
        const uint32_t valid = (32 * w + 32 <= NG) ? 0xffffffffu : ((1u << (NG - 32 * w)) - 1u);
        ob[0][q * W + w] = c2 & valid;
        ob[1][q * W + w] = c1 & valid;
    }
    // charges of this plane, in atom order: the first entry of each cell sums
    // that cell's entries in order
    const int c0 = cstart[(size_t)b * (NG + 1) + p], c1 = cstart[(size_t)b * (NG + 1) + p + 1];
    const int2 *qb = cq + (size_t)b * L.na;
    if constexpr (FIRST) {
        for (int e = c0 + tid; e < c1; e += blockDim.x) atomicMin(&first[qb[e].x], e);
        __syncthreads();
    }
    int2 *ql = qlist + ((size_t)b * NG + p) * NG * NG;
    for (int e = c0 + tid; e < c1; e += blockDim.x) {
        const int key = qb[e].x;
        if constexpr (FIRST) {
            if (first[key] != e) continue;
        } else {
            bool later = false;
            for (int f = c0; f < e && !later; ++f) later = qb[f].x == key;
            if (later) continue;
        }
        float acc = 0.f;
        for (int f = e; f < c1; ++f) {
            const int2 v = qb[f];
            if (v.x == key) acc = __fadd_rn(acc, __int_as_float(v.y));
        }
        ql[atomicAdd(&count, 1)] = make_int2(key, __float_as_int(acc));
    }
    uint32_t *dst = vbits + ((size_t)b * NG + p) * 2 * NG * W;
    for (int w = tid; w < 2 * NG * W; w += blockDim.x) dst[w] = (&ob[0][0])[w];
    __syncthreads();
    if (tid == 0) qcount[(size_t)b * NG + p] = count;
}

// ------------------------------------------------------------------ K1
// MODE 0: real part from the K0 bit planes + K0 charge list, store spectrum planes A.
// MODE 1: receptor grids (re, im) loaded from global, store spectrum planes A.
// MODE 2: like MODE 0 but store the voxel plane itself (ng x ng real and
//         imaginary parts) for parity checks; no FFT.
template <int N, int MODE>
__global__ void __launch_bounds__(kNT1, 1)
    k_plane_fwd(LigandView L, GridView G, const uint32_t *__restrict__ vbits, const int2 *__restrict__ qlist,
                const int *__restrict__ qcount, const float *__restrict__ src_r, const float *__restrict__ src_i,
                float2 *__restrict__ A, float *__restrict__ vox_r, float *__restrict__ vox_i) {
    constexpr int NG = N / 2, OFF = N / 4, PITCH = N + 1;
    constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
    constexpr int W = VoxShared<NG>::W;
    constexpr bool PR = prune_ok<N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *S = reinterpret_cast<float2 *>(smem_raw);   // N x PITCH

    const int p = blockIdx.x;
    const int b = blockIdx.y;
    const int tid = threadIdx.x;

    if constexpr (!PR && MODE != 2) {
        // unpruned passes read the padding: make it zero
        for (int c = tid; c < N * PITCH; c += blockDim.x) S[c] = make_float2(0.f, 0.f);
        __syncthreads();
    }
    if (MODE == 1) {
        for (int c = tid; c < NG * NG; c += blockDim.x) {
            const int q = c / NG, s = c % NG;
            const size_t gidx = ((size_t)p * NG + q) * NG + s;
            S[(q + OFF) * PITCH + s + OFF] = make_float2(src_r[gidx], src_i[gidx]);
        }
        __syncthreads();
    } else {
        const uint32_t *vb = vbits + ((size_t)b * NG + p) * 2 * NG * W;
        // compile-time trip count, both class words loaded unconditionally
        constexpr int CPT = (NG * NG + kNT1 - 1) / kNT1;
#pragma unroll
        for (int r = 0; r < CPT; ++r) {
            const int c = tid + r * kNT1;
            if (NG * NG % kNT1 == 0 || c < NG * NG) {
                const int q = c / NG, s = c % NG;
                const uint32_t bit = 1u << (s & 31);
                const uint32_t w2 = __ldg(&vb[q * W + (s >> 5)]), w1 = __ldg(&vb[NG * W + q * W + (s >> 5)]);
                const float v = (w2 & bit) ? L.delta : (w1 & bit) ? 1.0f : 0.0f;
                S[(q + OFF) * PITCH + s + OFF] = make_float2(v, 0.f);
            }
        }
        __syncthreads();
        const int nq = qcount[(size_t)b * NG + p];
        const int2 *ql = qlist + ((size_t)b * NG + p) * NG * NG;
        for (int e = tid; e < nq; e += blockDim.x) {
            const int2 c = ql[e];
            S[(c.x / NG + OFF) * PITCH + c.x % NG + OFF].y = __int_as_float(c.y);
        }
        __syncthreads();
        if (MODE == 2) {
            for (int c = tid; c < NG * NG; c += blockDim.x) {
                const int q = c / NG, s = c % NG;
                const float2 v = S[(q + OFF) * PITCH + s + OFF];
                const size_t gidx = (((size_t)b * NG + p) * NG + q) * NG + s;
                vox_r[gidx] = v.x;
                vox_i[gidx] = v.y;
            }
            return;
        }
    }

    // z-FFT of the NG non-zero rows (lanes = rows, pruned columns)
    for (int it = tid; it < NG * R2; it += blockDim.x) {
        const int t = it / NG, q = it % NG;
        fft_phase1<N, -1, PR>(S + (q + OFF) * PITCH, 1, t, G.tw);
    }
    __syncthreads();
    {
        constexpr int IPT = (NG * R1 + kNT1 - 1) / kNT1;
        float2 reg[IPT][R2];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = tid + r * kNT1;
            if (it < NG * R1) fft_phase2<N, -1>(S + ((it % NG) + OFF) * PITCH, 1, it / NG, reg[r]);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = tid + r * kNT1;
            if (it < NG * R1) {
                float2 *row = S + ((it % NG) + OFF) * PITCH;
                const int u = it / NG;
                static_for<0, R2>([&](auto k2) { row[u + R1 * k2] = reg[r][k2]; });
            }
        }
    }
    __syncthreads();
    // y-FFT of all N columns (lanes = columns, pruned rows); phase 2 -> global
    for (int it = tid; it < N * R2; it += blockDim.x) {
        const int t = it / N, c = it % N;
        fft_phase1<N, -1, PR>(S + c, PITCH, t, G.tw);
    }
    __syncthreads();
    float2 *Ab = A + ((size_t)b * NG + p) * N * N;
    for (int it = tid; it < N * R1; it += blockDim.x) {
        const int u = it / N, c = it % N;
        float2 o[R2];
        fft_phase2<N, -1>(S + c, PITCH, u, o);
        static_for<0, R2>([&](auto k2) { Ab[(size_t)(u + R1 * k2) * N + c] = o[k2]; });
    }
}

// K1, column-block form (MODE 0): the same forward plane transform with about
// half the shared memory, so two CTAs share an SM (used by the batched
// pipeline wherever two fit: N <= 128; B200 measurement at 12,800 rotations
// and 64 per launch: 6-10 % more rotations/s at N = 64..112, 0.6 % at 128,
// identical poses).  The z-FFT results of the
// NG non-zero rows stay resident (NG x (N+1)); the y-FFT then runs over
// blocks of CB columns through an N x (CB+1) buffer: pruned phase 1 from the
// resident rows into the block buffer, phase 2 from the block buffer
// straight to global memory.
constexpr int kNT1B = 512;

constexpr size_t kSmemMax = 227 * 1024;   // dynamic shared memory one CTA may hold

template <int N>
constexpr size_t fwd_cb_smem_of(int cb) {
    return ((size_t)(N / 2) * (N + 1) + (size_t)N * (cb + 1)) * sizeof(float2);
}

// Column-block width: 32 where it fits one CTA's shared memory, else 16 or 8.
template <int N>
constexpr int fwd_cb_width() {
    return fwd_cb_smem_of<N>(32) <= kSmemMax ? 32 : (fwd_cb_smem_of<N>(16) <= kSmemMax ? 16 : 8);
}

template <int N>
constexpr size_t fwd_cb_smem() {
    return fwd_cb_smem_of<N>(fwd_cb_width<N>());
}

// two CTAs and their 1 KB system reservations within the SM's 228 KB
template <int N>
constexpr bool fwd_cb_fits() {
    return fwd_cb_smem<N>() <= 113 * 1024;
}

// whether the one-CTA form's N x (N+1) plane fits one CTA (N <= 168); larger
// sizes run every mode in the column-block form
template <int N>
constexpr bool fwd_full_fits() {
    return (size_t)N * (N + 1) * sizeof(float2) <= kSmemMax;
}

// MODE as in k_plane_fwd: 0 ligand bits + charges, 1 receptor grids from
// global, 2 the voxel plane itself (no FFT).
template <int N, int MODE = 0>
__global__ void __launch_bounds__(kNT1B, fwd_cb_fits<N>() ? 2 : 1)
    k_plane_fwd_cb(LigandView L, GridView G, const uint32_t *__restrict__ vbits, const int2 *__restrict__ qlist,
                   const int *__restrict__ qcount, const float *__restrict__ src_r, const float *__restrict__ src_i,
                   float2 *__restrict__ A, float *__restrict__ vox_r, float *__restrict__ vox_i) {
    constexpr int NG = N / 2, OFF = N / 4, PZ = N + 1, CB = fwd_cb_width<N>(), PB = CB + 1;
    constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
    constexpr int W = VoxShared<NG>::W;
    constexpr bool PR = prune_ok<N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *Z = reinterpret_cast<float2 *>(smem_raw);   // NG rows x PZ
    float2 *Y = Z + NG * PZ;                             // N rows x PB
    const int p = blockIdx.x, b = blockIdx.y, tid = threadIdx.x;
    if constexpr (!PR && MODE != 2) {
        // the unpruned z pass reads the padding columns: make them zero
        for (int c = tid; c < NG * PZ; c += blockDim.x) Z[c] = make_float2(0.f, 0.f);
        __syncthreads();
    }

    // the plane's NG rows at column offset OFF (the pruned passes read no
    // other column)
    if constexpr (MODE == 1) {
        for (int c = tid; c < NG * NG; c += blockDim.x) {
            const int q = c / NG, s = c % NG;
            const size_t gidx = ((size_t)p * NG + q) * NG + s;
            Z[q * PZ + s + OFF] = make_float2(src_r[gidx], src_i[gidx]);
        }
        __syncthreads();
    } else {
        const uint32_t *vb = vbits + ((size_t)b * NG + p) * 2 * NG * W;
        // the cells of this thread with a compile-time trip count and both
        // class words loaded unconditionally: all loads in flight at once
        constexpr int CPT = (NG * NG + kNT1B - 1) / kNT1B;
#pragma unroll
        for (int r = 0; r < CPT; ++r) {
            const int c = tid + r * kNT1B;
            if (NG * NG % kNT1B == 0 || c < NG * NG) {
                const int q = c / NG, s = c % NG;
                const uint32_t bit = 1u << (s & 31);
                const uint32_t w2 = __ldg(&vb[q * W + (s >> 5)]), w1 = __ldg(&vb[NG * W + q * W + (s >> 5)]);
                const float v = (w2 & bit) ? L.delta : (w1 & bit) ? 1.0f : 0.0f;
                Z[q * PZ + s + OFF] = make_float2(v, 0.f);
            }
        }
        __syncthreads();
        const int nq = qcount[(size_t)b * NG + p];
        const int2 *ql = qlist + ((size_t)b * NG + p) * NG * NG;
        for (int e = tid; e < nq; e += blockDim.x) {
            const int2 c = ql[e];
            Z[(c.x / NG) * PZ + c.x % NG + OFF].y = __int_as_float(c.y);
        }
        __syncthreads();
        if constexpr (MODE == 2) {
            for (int c = tid; c < NG * NG; c += blockDim.x) {
                const int q = c / NG, s = c % NG;
                const float2 v = Z[q * PZ + s + OFF];
                const size_t gidx = (((size_t)b * NG + p) * NG + q) * NG + s;
                vox_r[gidx] = v.x;
                vox_i[gidx] = v.y;
            }
            return;
        }
    }
    // z-FFT of the NG rows (lanes = rows, pruned columns)
    for (int it = tid; it < NG * R2; it += blockDim.x) {
        const int t = it / NG, q = it % NG;
        fft_phase1<N, -1, PR>(Z + q * PZ, 1, t, G.tw);
    }
    __syncthreads();
    {
        constexpr int IPT = (NG * R1 + kNT1B - 1) / kNT1B;
        float2 reg[IPT][R2];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = tid + r * kNT1B;
            if (it < NG * R1) fft_phase2<N, -1>(Z + (it % NG) * PZ, 1, it / NG, reg[r]);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = tid + r * kNT1B;
            if (it < NG * R1) {
                float2 *row = Z + (it % NG) * PZ;
                const int u = it / NG;
                static_for<0, R2>([&](auto k2) { row[u + R1 * k2] = reg[r][k2]; });
            }
        }
    }
    __syncthreads();
    // y-FFT of the N columns, CB at a time
    float2 *Ab = A + ((size_t)b * NG + p) * N * N;
    for (int cb = 0; cb < N; cb += CB) {
        for (int it = tid; it < CB * R2; it += blockDim.x) {
            const int t = it / CB, c = it % CB;
            if (cb + c >= N) continue;
            float2 v[R1];
            static_for<0, R1>([&](auto m_) {
                constexpr int m = decltype(m_)::value;
                if constexpr (PR) {
                    if constexpr (m < R1 / 4 || m >= 3 * R1 / 4) {
                        v[m] = make_float2(-0.f, -0.f);
                    } else {
                        v[m] = Z[(t + R2 * (m - R1 / 4)) * PZ + cb + c];   // row n - OFF, n = t + R2 m
                    }
                } else {
                    const int q = t + R2 * m - OFF;   // resident row of y = t + R2 m, if any
                    v[m] = ((unsigned)q < (unsigned)NG) ? Z[q * PZ + cb + c] : make_float2(0.f, 0.f);
                }
            });
            Dft<R1, -1>::run(v);
            static_for<0, R1>([&](auto k1_) {
                constexpr int k1 = decltype(k1_)::value;
                float2 x = v[k1];
                if constexpr (k1 != 0) x = cmul(x, __ldg(&G.tw[t * k1]));
                Y[(k1 * R2 + t) * PB + c] = x;
            });
        }
        __syncthreads();
        for (int it = tid; it < CB * R1; it += blockDim.x) {
            const int u = it / CB, c = it % CB;
            if (cb + c >= N) continue;
            float2 o[R2];
            fft_phase2<N, -1>(Y + c, PB, u, o);
            static_for<0, R2>([&](auto k2) { Ab[(size_t)(u + R1 * k2) * N + cb + c] = o[k2]; });
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ K2 (receptor)
// Forward x-FFT of the ng non-zero spectrum planes of the receptor: writes the
// full receptor spectrum R^[kx][ky][kz].  CTA = (ky, 32 kz lines); the last
// tile is partial when N is not a multiple of 32.
template <int N>
__global__ void __launch_bounds__(kNT)
    k_xline_rec(GridView G, const float2 *__restrict__ A, float2 *__restrict__ Rh) {
    constexpr int NG = N / 2, OFF = N / 4;
    constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
    constexpr int TILES = (N + kLT - 1) / kLT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *X = reinterpret_cast<float2 *>(smem_raw);   // N x kLT
    constexpr bool PR = prune_ok<N>();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int ky = blockIdx.x / TILES;
    const int kz = (blockIdx.x % TILES) * kLT + lane;
    const bool ok = kz < N;
    if constexpr (!PR) {
        for (int c = threadIdx.x; c < N * kLT; c += blockDim.x) X[c] = make_float2(0.f, 0.f);
        __syncthreads();
    }
    for (int pp = warp; pp < NG; pp += nwarp)
        X[(pp + OFF) * kLT + lane] = ok ? A[((size_t)pp * N + ky) * N + kz] : make_float2(0.f, 0.f);
    __syncthreads();
    for (int it = threadIdx.x; it < kLT * R2; it += blockDim.x)
        fft_phase1<N, -1, PR>(X + (it % kLT), kLT, it / kLT, G.tw);
    __syncthreads();
    for (int it = threadIdx.x; it < kLT * R1; it += blockDim.x) {
        const int ln = it % kLT, u = it / kLT;
        float2 o[R2];
        fft_phase2<N, -1>(X + ln, kLT, u, o);
        if (ok)
            static_for<0, R2>([&](auto k2) { Rh[((size_t)(u + R1 * k2) * N + ky) * N + kz] = o[k2]; });
    }
}

// ------------------------------------------------------------------ K2 (docking)
// The score grid s = IFFT(conj(R^) L^) is real, so only its Hermitian part
//   H(k) = (P(k) + conj(P(-k))) / 2,   P = conj(R^) L^,
// contributes: IFFT(H) = Re(IFFT(P)) exactly.  This kernel keeps the rows
// ky in [1, N/2) of the x-inverted H and packs the two self-conjugate rows
// ky = 0 and ky = N/2 into row 0 (row0 = g(ky=0) + i g(ky=N/2)); both become
// real after the inverse along kz, so the plane kernel can unpack them.
//
// CTA = (ky in [0, N/2), 32 kz lines).  Per pass it loads the own tile
// (ky, kz) and the mirror tile (-ky, -kz) straight from global memory into
// the pruned forward x-FFT, multiplies both by conj(R^), folds the mirror into
// H and runs the inverse x-FFT of the own tile.  CTAs of row 0 run two passes
// (ky = 0 and ky = N/2) and pack them.  Output Gh[x][ky][kz], ky < N/2.
// LT kz lines per CTA (the tile shape the autotuner picks: 8, 16 or 32), 16 LT
// threads, xline_occ<N>() / LT CTAs per SM (below).
//
// xline_occ: threads per SM the kernel is compiled for, in units of 16:
// 1,280 where that register budget (51 per thread) holds the kernel without
// spills, 512 above N = 160 (radices up to 20 need the registers), else 1,024.
// B200, 13,824 rotations at 192 per launch: +2.0 % at N=96; with spills at
// N=112 it lost 2 %.  N = 128 runs 1,280 since its first-pass loads are issued
// ahead of the DFTs and its twiddles come from shared memory (xline_tw_smem).
template <int N>
constexpr int xline_occ() {
    return (N == 32 || N == 64 || N == 72 || N == 80 || N == 96 || N == 128) ? 80 : (N > 160 ? 32 : 64);
}

// Twiddles of the x-line kernel from shared memory instead of the read-only
// cache.  Measured at N = 128 (B200, 54,000 rotations, 192 per launch): with
// five 256-thread CTAs per SM (48 registers) 267 ms per step for this kernel,
// against 277 ms with cached loads and 278 ms at four CTAs per SM; at four
// CTAs per SM the shared-memory table lost (285 ms).  Other sizes keep the
// cached loads.
template <int N>
constexpr bool xline_tw_smem() {
    return N == 128;
}

// Block order of the x-line kernels.  Every launch-group rotation reads the
// same receptor spectrum tiles, which stay in L2 across the launch while the
// spectrum fits (16 MiB at N = 128); above N = 224 it does not (8 N^3 bytes,
// 134 MB at N = 256), so the rotation becomes the fastest-varying block index
// and the launch's rotations read each (ky, kz-tile) of R^ back to back from
// L2 instead of streaming all of it from HBM once per rotation.
template <int N>
constexpr bool xline_rot_fast() {
    return N > 224;
}
template <int N>
__device__ __forceinline__ void xline_block(int &tile_id, int &b) {
    if constexpr (xline_rot_fast<N>()) {
        tile_id = blockIdx.y;
        b = blockIdx.x;
    } else {
        tile_id = blockIdx.x;
        b = blockIdx.y;
    }
}
template <int N>
inline dim3 xline_grid(int tiles, int nb) {
    return xline_rot_fast<N>() ? dim3(nb, tiles) : dim3(tiles, nb);
}

// Shared memory of k_xline_herm: the own and mirror tiles, and the twiddle
// table where xline_tw_smem<N>().
template <int N, int LT>
constexpr size_t xline_smem() {
    return (size_t)(2 * N * LT + (xline_tw_smem<N>() ? N : 0)) * sizeof(float2);
}
// Whether an LT-line tile fits one CTA's 227 KB (32-line tiles stop at N = 450;
// above, a request for them runs 16-line tiles).
template <int N, int LT>
constexpr bool xline_tile_fits() {
    return xline_smem<N, LT>() <= 227 * 1024;
}

template <int N, int LT = kLT>
__global__ void __launch_bounds__(16 * LT, xline_occ<N>() / LT)
    k_xline_herm(GridView G, const float2 *__restrict__ A, const float2 *__restrict__ Rh, float2 *__restrict__ Gh) {
    constexpr int NG = N / 2, NH = N / 2, OFF = N / 4;
    constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
    constexpr bool PR = prune_ok<N>();
    constexpr int TILES = (N + LT - 1) / LT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *X0 = reinterpret_cast<float2 *>(smem_raw);   // own tile   [N][LT]
    float2 *X1 = X0 + N * LT;                           // mirror tile [N][LT]
    constexpr int NT = 16 * LT;
    float2 *TWs = X1 + N * LT;                          // twiddles W_N^j (xline_tw_smem)
    if constexpr (xline_tw_smem<N>()) {
        for (int e = threadIdx.x; e < N; e += NT) TWs[e] = __ldg(&G.tw[e]);
        __syncthreads();
    }
    auto tw_at = [&](int j) {
        if constexpr (xline_tw_smem<N>()) return TWs[j];
        else return __ldg(&G.tw[j]);
    };
    const int lane = threadIdx.x % LT;
    int tile_id, b;
    xline_block<N>(tile_id, b);
    const int ky = tile_id / TILES;
    const int kz = (tile_id % TILES) * LT + lane;
    const bool ok = kz < N;
    const int kzm = (N - kz) % N;
    const float2 *Ab = A + (size_t)b * NG * N * N;
    float2 *Gb = Gh + (size_t)b * N * NH * N;
    const int passes = (ky == 0) ? 2 : 1;

    for (int pass = 0; pass < passes; ++pass) {
        const int kyo = pass == 0 ? ky : NH;   // own row
        const int kym = (N - kyo) % N;         // mirror row
        // forward x pass 1 on both tiles, straight from global (pruned rows):
        // every item of this thread issues its loads before the first DFT, so
        // the HBM latency is paid once per thread, not once per item
        constexpr int IT1 = (2 * LT * R2 + NT - 1) / NT;
        float2 v1[IT1][R1];
#pragma unroll
        for (int r = 0; r < IT1; ++r) {
            const int it = threadIdx.x + r * NT;
            const int s = it / (LT * R2);
            const int t = (it / LT) % R2;
            const int row = s ? kym : kyo, col = s ? kzm : kz;
            const bool live = ok && it < 2 * LT * R2;
            static_for<0, R1>([&](auto m_) {
                constexpr int mm = decltype(m_)::value;
                const int pp = t + R2 * mm - OFF;   // spectrum plane of x = t + R2 mm, if any
                if constexpr (PR && (mm < R1 / 4 || mm >= 3 * R1 / 4)) {
                    v1[r][mm] = make_float2(-0.f, -0.f);
                } else if constexpr (PR) {
                    v1[r][mm] = live ? Ab[((size_t)pp * N + row) * N + col] : make_float2(0.f, 0.f);
                } else {
                    v1[r][mm] = (live && (unsigned)pp < (unsigned)NG) ? Ab[((size_t)pp * N + row) * N + col]
                                                                     : make_float2(0.f, 0.f);
                }
            });
        }
#pragma unroll
        for (int r = 0; r < IT1; ++r) {
            const int it = threadIdx.x + r * NT;
            if (it < 2 * LT * R2) {
                const int s = it / (LT * R2);
                const int t = (it / LT) % R2;
                Dft<R1, -1>::run(v1[r]);
                float2 *X = s ? X1 : X0;
                static_for<0, R1>([&](auto k1_) {
                    constexpr int k1 = decltype(k1_)::value;
                    float2 x = v1[r][k1];
                    if constexpr (k1 != 0) x = cmul(x, tw_at(t * k1));
                    X[(k1 * R2 + t) * LT + lane] = x;
                });
            }
        }
        __syncthreads();
        // forward x pass 2 and the conj(R^) product, held in registers
        constexpr int IPT = (2 * LT * R1 + NT - 1) / NT;
        float2 reg[IPT][R2];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = threadIdx.x + r * NT;
            if (it < 2 * LT * R1) {
                const int s = it / (LT * R1);
                const int u = (it / LT) % R1;
                const int row = s ? kym : kyo, col = s ? kzm : kz;
                fft_phase2<N, -1>((s ? X1 : X0) + lane, LT, u, reg[r]);
                static_for<0, R2>([&](auto k2) {
                    const int kx = u + R1 * k2;
                    const float2 rh = ok ? __ldg(&Rh[((size_t)kx * N + row) * N + col]) : make_float2(0.f, 0.f);
                    reg[r][k2] = cmulconj(rh, reg[r][k2]);
                });
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = threadIdx.x + r * NT;
            if (it < 2 * LT * R1) {
                const int s = it / (LT * R1);
                const int u = (it / LT) % R1;
                float2 *X = s ? X1 : X0;
                static_for<0, R2>([&](auto k2) { X[(u + R1 * k2) * LT + lane] = reg[r][k2]; });
            }
        }
        __syncthreads();
        // inverse x pass 1 of H = (P_own(kx) + conj(P_mirror(-kx))) / 2, in place in X0
        for (int it = threadIdx.x; it < LT * R2; it += blockDim.x) {
            const int t = it / LT;
            float2 v[R1];
            static_for<0, R1>([&](auto m_) {
                constexpr int mm = decltype(m_)::value;
                const int e = t + R2 * mm;
                const float2 a = X0[e * LT + lane];
                const float2 c = X1[((N - e) % N) * LT + lane];
                v[mm] = make_float2(0.5f * (a.x + c.x), 0.5f * (a.y - c.y));
            });
            Dft<R1, +1>::run(v);
            static_for<0, R1>([&](auto k1_) {
                constexpr int k1 = decltype(k1_)::value;
                float2 x = v[k1];
                if constexpr (k1 != 0) x = cmul(x, conjf2(tw_at(t * k1)));
                X0[(k1 * R2 + t) * LT + lane] = x;
            });
        }
        __syncthreads();
        // inverse x pass 2 -> Gh (row 0 packs ky = 0 and ky = N/2)
        for (int it = threadIdx.x; it < LT * R1; it += blockDim.x) {
            const int u = it / LT;
            float2 o[R2];
            fft_phase2<N, +1>(X0 + lane, LT, u, o);
            if (ok) {
                static_for<0, R2>([&](auto k2) {
                    const int x = u + R1 * k2;
                    float2 *dst = &Gb[((size_t)x * NH + ky) * N + kz];
                    if (ky != 0 || pass == 0) {
                        *dst = o[k2];
                    } else {
                        // same thread wrote the ky = 0 value in pass 0
                        const float2 g0 = *dst;
                        *dst = make_float2(g0.x - o[k2].y, g0.y + o[k2].x);
                    }
                });
            }
        }
        __syncthreads();
    }
}

// K2, register-fold form.  The same transform as k_xline_herm with the
// forward split reversed (pass 1 a DFT-F1 over stride F2, pass 2 a DFT-F2
// whose outputs sit at kx = u + F1 k2): the conjugate partner -kx of every
// output of the own item u is an output of the mirror item (F1 - u) mod F1,
// so one thread transforms both, multiplies both by conj(R^), folds them into
// H in registers, and runs the first inverse pass (a DFT-F2 over the same
// stride F1, the inverse split being F2 x F1) before anything is stored.  The
// mirror tile's products never go back to shared memory, and the fold and
// the first inverse pass need no barrier of their own: three barriers per
// pass instead of five.
template <int N>
struct FoldPlan {
    static constexpr int F1 = Plan<N>::R2, F2 = Plan<N>::R1;
};
// Used for the 16-line tiles at N = 128, compiled for four 256-thread CTAs
// per SM (64 registers).  B200, 13,824 of the 54,000 rotations at 512 per
// launch: 237.4 ms per 54,000 rotations against 262.8 for k_xline_herm; at
// five CTAs per SM (48 registers, 100 bytes of spills) 284.0, at three 267.2.
template <int N>
constexpr bool xline_fold_ok() {
    return N == 128;
}
template <int N>
constexpr int xline_fold_occ() {
    return 64;
}

template <int N, int LT = kLT>
__global__ void __launch_bounds__(16 * LT, xline_fold_occ<N>() / LT)
    k_xline_fold(GridView G, const float2 *__restrict__ A, const float2 *__restrict__ Rh, float2 *__restrict__ Gh) {
    constexpr int NG = N / 2, NH = N / 2, OFF = N / 4;
    constexpr int F1 = FoldPlan<N>::F1, F2 = FoldPlan<N>::F2;
    constexpr bool PR = N % 4 == 0 && F1 % 4 == 0;
    constexpr int TILES = (N + LT - 1) / LT;
    constexpr int NT = 16 * LT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *X0 = reinterpret_cast<float2 *>(smem_raw);   // own tile   [N][LT]
    float2 *X1 = X0 + N * LT;                           // mirror tile [N][LT]
    float2 *TWs = X1 + N * LT;                          // twiddles W_N^j (xline_tw_smem)
    if constexpr (xline_tw_smem<N>()) {
        for (int e = threadIdx.x; e < N; e += NT) TWs[e] = __ldg(&G.tw[e]);
        __syncthreads();
    }
    auto tw_at = [&](int j) {
        if constexpr (xline_tw_smem<N>()) return TWs[j];
        else return __ldg(&G.tw[j]);
    };
    const int lane = threadIdx.x % LT;
    int tile_id, b;
    xline_block<N>(tile_id, b);
    const int ky = tile_id / TILES;
    const int kz = (tile_id % TILES) * LT + lane;
    const bool ok = kz < N;
    const int kzm = (N - kz) % N;
    const float2 *Ab = A + (size_t)b * NG * N * N;
    float2 *Gb = Gh + (size_t)b * N * NH * N;
    const int passes = (ky == 0) ? 2 : 1;

    for (int pass = 0; pass < passes; ++pass) {
        const int kyo = pass == 0 ? ky : NH;   // own row
        const int kym = (N - kyo) % N;         // mirror row
        // forward pass 1 (DFT-F1 over stride F2) on both tiles, straight from
        // global (pruned rows), every load of a thread issued before its DFTs
        constexpr int IT1 = (2 * LT * F2 + NT - 1) / NT;
        float2 v1[IT1][F1];
#pragma unroll
        for (int r = 0; r < IT1; ++r) {
            const int it = threadIdx.x + r * NT;
            const int s = it / (LT * F2);
            const int t = (it / LT) % F2;
            const int row = s ? kym : kyo, col = s ? kzm : kz;
            const bool live = ok && it < 2 * LT * F2;
            static_for<0, F1>([&](auto m_) {
                constexpr int mm = decltype(m_)::value;
                const int pp = t + F2 * mm - OFF;   // spectrum plane of x = t + F2 mm, if any
                if constexpr (PR && (mm < F1 / 4 || mm >= 3 * F1 / 4)) {
                    v1[r][mm] = make_float2(-0.f, -0.f);
                } else if constexpr (PR) {
                    v1[r][mm] = live ? Ab[((size_t)pp * N + row) * N + col] : make_float2(0.f, 0.f);
                } else {
                    v1[r][mm] = (live && (unsigned)pp < (unsigned)NG) ? Ab[((size_t)pp * N + row) * N + col]
                                                                     : make_float2(0.f, 0.f);
                }
            });
        }
#pragma unroll
        for (int r = 0; r < IT1; ++r) {
            const int it = threadIdx.x + r * NT;
            if (it < 2 * LT * F2) {
                const int s = it / (LT * F2);
                const int t = (it / LT) % F2;
                Dft<F1, -1>::run(v1[r]);
                float2 *X = s ? X1 : X0;
                static_for<0, F1>([&](auto k1_) {
                    constexpr int k1 = decltype(k1_)::value;
                    float2 x = v1[r][k1];
                    if constexpr (k1 != 0) x = cmul(x, tw_at(t * k1));
                    X[(k1 * F2 + t) * LT + lane] = x;
                });
            }
        }
        __syncthreads();
        // forward pass 2 of the own item u and the mirror item (F1 - u) mod F1,
        // conj(R^) products, H = (P_own(kx) + conj P_mirror(-kx)) / 2 and the
        // first inverse pass, in registers
        constexpr int IT2 = (LT * F1 + NT - 1) / NT;
        float2 h[IT2][F2];
#pragma unroll
        for (int r = 0; r < IT2; ++r) {
            const int it = threadIdx.x + r * NT;
            if (it < LT * F1) {
                const int u = it / LT;
                const int um = (F1 - u) % F1;
                float2 pm[F2];
                static_for<0, F2>([&](auto n2_) {
                    constexpr int n2 = decltype(n2_)::value;
                    h[r][n2] = X0[(u * F2 + n2) * LT + lane];
                    pm[n2] = X1[(um * F2 + n2) * LT + lane];
                });
                Dft<F2, -1>::run(h[r]);
                Dft<F2, -1>::run(pm);
                static_for<0, F2>([&](auto k2_) {
                    constexpr int k2 = decltype(k2_)::value;
                    const float2 rov = ok ? __ldg(&Rh[((size_t)(u + F1 * k2) * N + kyo) * N + kz]) : make_float2(0.f, 0.f);
                    const float2 rm = ok ? __ldg(&Rh[((size_t)(um + F1 * k2) * N + kym) * N + kzm]) : make_float2(0.f, 0.f);
                    h[r][k2] = cmulconj(rov, h[r][k2]);
                    pm[k2] = cmulconj(rm, pm[k2]);
                });
                // the partner of kx = u + F1 k2 is mirror output (F2 - 1 - k2)
                // for u > 0 and (F2 - k2) mod F2 for u = 0
                if (u == 0) {
                    static_for<0, F2>([&](auto k2_) {
                        constexpr int k2 = decltype(k2_)::value, j2 = (F2 - k2) % F2;
                        h[r][k2] = make_float2(0.5f * (h[r][k2].x + pm[j2].x), 0.5f * (h[r][k2].y - pm[j2].y));
                    });
                } else {
                    static_for<0, F2>([&](auto k2_) {
                        constexpr int k2 = decltype(k2_)::value, j2 = F2 - 1 - k2;
                        h[r][k2] = make_float2(0.5f * (h[r][k2].x + pm[j2].x), 0.5f * (h[r][k2].y - pm[j2].y));
                    });
                }
                Dft<F2, +1>::run(h[r]);
                static_for<1, F2>([&](auto k1_) {
                    constexpr int k1 = decltype(k1_)::value;
                    h[r][k1] = cmul(h[r][k1], conjf2(tw_at(u * k1)));
                });
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < IT2; ++r) {
            const int it = threadIdx.x + r * NT;
            if (it < LT * F1) {
                const int u = it / LT;
                static_for<0, F2>([&](auto k1) { X0[(k1 * F1 + u) * LT + lane] = h[r][k1]; });
            }
        }
        __syncthreads();
        // inverse pass 2 (DFT-F1 over items u2 < F2) -> Gh (row 0 packs ky = 0 and ky = N/2)
        for (int it = threadIdx.x; it < LT * F2; it += NT) {
            const int u2 = it / LT;
            float2 o[F1];
            static_for<0, F1>([&](auto n2) { o[decltype(n2)::value] = X0[(u2 * F1 + decltype(n2)::value) * LT + lane]; });
            Dft<F1, +1>::run(o);
            if (ok) {
                static_for<0, F1>([&](auto k2) {
                    const int x = u2 + F2 * k2;
                    float2 *dst = &Gb[((size_t)x * NH + ky) * N + kz];
                    if (ky != 0 || pass == 0) {
                        *dst = o[k2];
                    } else {
                        // same thread wrote the ky = 0 value in pass 0
                        const float2 g0 = *dst;
                        *dst = make_float2(g0.x - o[k2].y, g0.y + o[k2].x);
                    }
                });
            }
        }
        if (passes > 1) __syncthreads();
    }
}

// ------------------------------------------------------------------ K3
// Selection order for top-t: larger key first, then smaller linear index.
// NaN keys are never selected (they fail every comparison in the reference).
__device__ __forceinline__ bool key_better(float a, int ia, float b, int ib) {
    return (a > b) || (a == b && ia < ib);
}

struct Cand {
    float key;
    int idx;
};

// Order-preserving integer image of a key for the warp reductions of the
// plane kernel (redux.sync reduces integers in one instruction where a
// shuffle tree takes five dependent steps): larger keys map to larger
// integers, -0 and +0 to the same one (they compare equal), NaN below every
// key.
__device__ __forceinline__ int key_ord(float k) {
    if (k != k) return INT_MIN;
    const int b = __float_as_int(k == 0.f ? 0.f : k);
    return b >= 0 ? b : b ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float ord_key(int o) {
    return __int_as_float(o >= 0 ? o : o ^ 0x7FFFFFFF);
}

// The best candidate of a warp's lanes in selection order (larger key, then
// smaller cell index; the lanes' cell indices are distinct), broadcast to
// every lane, and the lane that holds it; idx < 0 when no lane holds one.
// The largest key comes from one integer reduction over the keys'
// order-preserving images, the smallest index among its holders from a
// second.
__device__ __forceinline__ Cand warp_best(Cand c, int &owner) {
    const bool valid = c.idx >= 0;
    const int ko = valid ? key_ord(c.key) : INT_MIN;
    const int kmax = __reduce_max_sync(0xffffffffu, ko);
    const bool tie = valid && ko == kmax;
    const int imin = __reduce_min_sync(0xffffffffu, tie ? c.idx : INT_MAX);
    const unsigned win = __ballot_sync(0xffffffffu, tie && c.idx == imin);
    if (win == 0) {
        owner = 0;
        return Cand{0.f, -1};
    }
    owner = __ffs(win) - 1;
    return Cand{__shfl_sync(0xffffffffu, c.key, owner), imin};
}

// Block-wide best candidate; idx < 0 means "none".
__device__ __forceinline__ Cand block_best(Cand mine, Cand *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int owner;
    mine = warp_best(mine, owner);
    if (lane == 0) red[warp] = mine;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        const Cand c = warp_best((lane < nw) ? red[lane] : Cand{0.f, -1}, owner);
        if (lane == 0) red[32] = c;
    }
    __syncthreads();
    const Cand r = red[32];
    __syncthreads();
    return r;
}

// Per-thread sorted list of the T best (key, index) pairs seen, best first.
// Empty slots hold (-inf, INT_MAX), which every non-NaN key beats, so the
// one test against the last slot rejects NaN, too-small keys and equal keys
// of later cells alike; an accepted key enters through a branch-free
// compare-and-select network (the list is sorted, so "beats slot j" implies
// "beats slot j+1").  Only candidates strictly after `floor` in selection
// order are kept (used when a plane's top-t is found in several passes of T).
template <int T>
struct TopList {
    float k[T];
    int i[T];
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int j = 0; j < T; ++j) {
            k[j] = -INFINITY;
            i[j] = INT_MAX;
        }
    }
    // FLOOR: a floor from an earlier pass is in force (uniform per launch).
    template <bool FLOOR = true>
    __device__ __forceinline__ void insert(float key, int idx, const Cand &floor) {
        if (!((key > k[T - 1]) | ((key == k[T - 1]) & (idx < i[T - 1])))) return;
        if (FLOOR && floor.idx >= 0 && !key_better(floor.key, floor.idx, key, idx)) return;
        bool b[T];
#pragma unroll
        for (int j = 0; j < T; ++j) b[j] = (key > k[j]) | ((key == k[j]) & (idx < i[j]));
#pragma unroll
        for (int j = T - 1; j >= 1; --j) {
            k[j] = b[j - 1] ? k[j - 1] : (b[j] ? key : k[j]);
            i[j] = b[j - 1] ? i[j - 1] : (b[j] ? idx : i[j]);
        }
        k[0] = b[0] ? key : k[0];
        i[0] = b[0] ? idx : i[0];
    }
    // the best entry as a candidate (index -1 when the list is empty)
    __device__ __forceinline__ Cand head() const { return Cand{k[0], i[0] == INT_MAX ? -1 : i[0]}; }
    __device__ __forceinline__ void pop() {
#pragma unroll
        for (int j = 0; j < T - 1; ++j) {
            k[j] = k[j + 1];
            i[j] = i[j + 1];
        }
        k[T - 1] = -INFINITY;
        i[T - 1] = INT_MAX;
    }
};

// K3: one x-plane of one rotation.  Input Gh[x][ky < N/2][kz] from
// k_xline_herm.  (1) inverse FFT along kz of the N/2 rows, straight from
// global memory; row 0 then holds h0 + i h_{N/2}, both real.  (2) complex-to-
// real inverse along ky for every z column: with X the half spectrum,
//   Z[k] = (X[k] + conj X[N/2-k]) + i w^k (X[k] - conj X[N/2-k]),  w = e^{2 pi i/N},
// the N/2-point inverse FFT of Z gives s[2m] + i s[2m+1].  The scores feed a
// per-thread top-T list directly (no score store), then a block merge writes
// this plane's candidates cand[(b*N + x)*t + out0 + j] for j < nsel.
// Keys are raw scores: ordering by raw equals ordering by raw / nf3 (a
// positive constant), so the merge kernel divides only the winners.
// Radix plans of this kernel, chosen per context by the autotuner: variant 0
// uses the line plans of N (kz) and N/2 (ky), variant 1 reverses the kz split
// (R2 x R1), variant 2 the ky split.  Three CTAs per SM (<= 42 registers)
// where the radices are small enough.
constexpr int kC2RPlans = 3;
template <int N, int V>
struct C2RPlan {
    static constexpr int R1 = V == 1 ? Plan<N>::R2 : Plan<N>::R1;
    static constexpr int R2 = V == 1 ? Plan<N>::R1 : Plan<N>::R2;
    static constexpr int Q1 = V == 2 ? Plan<N / 2>::R2 : Plan<N / 2>::R1;
    static constexpr int Q2 = V == 2 ? Plan<N / 2>::R1 : Plan<N / 2>::R2;
};

// Shared memory of k_plane_c2r: the N/2 x PITCH plane.
template <int N, int V>
constexpr size_t c2r_smem() {
    constexpr size_t PA = N + C2RPlan<N, V>::R1, PB = N + 8;
    return (size_t)(N / 2) * (PA > PB ? PA : PB) * sizeof(float2);
}

// Whether the plane kernel folds the half spectrum inside pass 1 of its ky
// transform (both splits of the ky axis even).
template <int N, int V>
constexpr bool c2r_fold_ok() {
    return N == 128 && C2RPlan<N, V>::Q1 % 2 == 0 && C2RPlan<N, V>::Q2 % 2 == 0;
}

template <int N, int T, int V = 0>
constexpr int c2r_min_blocks() {
    using P = C2RPlan<N, V>;
    constexpr size_t pitch = (size_t)N + (P::R1 > 8 ? P::R1 : 8);
    if ((size_t)(N / 2) * pitch * 8 > 113 * 1024) return 1;   // one CTA per SM by shared memory
    return (T <= 4 && P::R1 <= 8 && P::R2 <= 16 && P::Q1 <= 8 && P::Q2 <= 16) ? 3 : 2;
}

// The plane kernel's item loops: items tid, tid + kNT, ... below COUNT, with
// a compile-time trip count (blockDim.x is always kNT here) so that each loop
// unrolls (3.4 % less time for this kernel at N = 128 than the runtime-bounded
// loops).
#define MDB_K3_ITEMS(it, COUNT)                                                                 \
    _Pragma("unroll") for (int r_##it = 0; r_##it < ((COUNT) + kNT - 1) / kNT; ++r_##it)       \
        if (const int it = tid + r_##it * kNT; ((COUNT) % kNT == 0) || it < (COUNT))

template <int N, int T, int V = 0>
__global__ void __launch_bounds__(kNT, c2r_min_blocks<N, T, V>())
    k_plane_c2r(GridView G, const float2 *__restrict__ Gh, int t, float nf3f, int out0, int nsel,
                Cand *__restrict__ cand) {
    constexpr int NH = N / 2;
    constexpr int R1 = C2RPlan<N, V>::R1, R2 = C2RPlan<N, V>::R2;
    constexpr int Q1 = C2RPlan<N, V>::Q1, Q2 = C2RPlan<N, V>::Q2;
    constexpr int PA = N + N / R2;   // step-1 layout: one pad per R2 block
    constexpr int PB = N + 8;        // step-2 layout (natural order)
    constexpr int PITCH = PA > PB ? PA : PB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *S = reinterpret_cast<float2 *>(smem_raw);   // NH x PITCH
    auto tw_at = [&](int j) { return __ldg(&G.tw[j]); };
    const int x = blockIdx.x;
    const int b = blockIdx.y;
    const int tid = threadIdx.x;
    const float2 *Gp = Gh + ((size_t)b * N + x) * NH * N;

    // The z pass works on whole rows.  Where the rows split evenly over the
    // warps (WZ), warp w owns rows [w NH/16, (w+1) NH/16) in both of its
    // passes, so the passes are separated by warp barriers only; the plane
    // barrier comes once, before the ky pass reads across rows.
    constexpr bool WZ = kNT == 512 && NH % 16 == 0 && (NH / 16 * R2) % 32 == 0 && (NH / 16 * R1) % 32 == 0;
    // (1a) inverse kz pass 1, straight from global: item = (row, t), t fastest
    auto z_pass1 = [&](int it) {
        const int row = it / R2, t = it % R2;
        float2 v[R1];
        static_for<0, R1>([&](auto m_) {
            constexpr int mm = decltype(m_)::value;
            v[mm] = __ldg(&Gp[(size_t)row * N + t + R2 * mm]);
        });
        Dft<R1, +1>::run(v);
        static_for<0, R1>([&](auto k1_) {
            constexpr int k1 = decltype(k1_)::value;
            float2 xv = v[k1];
            if constexpr (k1 != 0) xv = cmul(xv, conjf2(tw_at(t * k1)));
            S[row * PITCH + k1 * (R2 + 1) + t] = xv;
        });
    };
    if constexpr (WZ) {
        constexpr int IPW = NH / 16 * R2;
#pragma unroll
        for (int r = 0; r < IPW / 32; ++r) z_pass1((tid >> 5) * IPW + (tid & 31) + 32 * r);
        __syncwarp();
    } else {
        MDB_K3_ITEMS(it, NH * R2) { z_pass1(it); }
        __syncthreads();
    }
    // (1b) inverse kz pass 2: item = (row, u), u fastest; natural order after a barrier
    {
        constexpr int IPW = WZ ? NH / 16 * R1 : 0;
        constexpr int IPT = WZ ? IPW / 32 : (NH * R1 + kNT - 1) / kNT;
        auto item = [&](int r) { return WZ ? (tid >> 5) * IPW + (tid & 31) + 32 * r : tid + r * kNT; };
        float2 reg[IPT][R2];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = item(r);
            if (WZ || it < NH * R1) {
                const int row = it / R1, u = it % R1;
                static_for<0, R2>([&](auto n2_) {
                    constexpr int n2 = decltype(n2_)::value;
                    reg[r][n2] = S[row * PITCH + u * (R2 + 1) + n2];
                });
                Dft<R2, +1>::run(reg[r]);
            }
        }
        if constexpr (WZ) __syncwarp();
        else __syncthreads();
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = item(r);
            if (WZ || it < NH * R1) {
                const int row = it / R1, u = it % R1;
                static_for<0, R2>([&](auto k2) { S[row * PITCH + u + R1 * k2] = reg[r][k2]; });
            }
        }
    }
    __syncthreads();
    if constexpr (c2r_fold_ok<N, V>()) {
        // (2a + 2b) the fold into Z and pass 1 of the N/2-point inverse along
        // ky in one item.  Pass 1 item tt reads and writes the rows
        // tt + Q2 m; the fold partner N/2 - k of row k = tt + Q2 m is row
        // (Q2 - tt) + Q2 (Q1 - 1 - m) for tt > 0, so item g takes the row
        // sets tt = g and Q2 - g, and item 0 the two sets that pair with
        // themselves (tt = 0: Q2 m with Q2 (Q1 - m), row 0 packed; tt = Q2/2).
        // Each item reads and writes only its own rows: no barrier between
        // the fold and the pass.
        // Z_k = E + i w^k D, E = a + conj c, D = a - conj c, a = X_k, c = X_{N/2-k};
        // w^{N/2-k} = -conj(w^k).  The folded rows go back to their own slots
        // (eight values in registers at a time, which keeps the kernel at 40
        // registers without spills) and each row set is then reloaded for its
        // DFT; the empty asm statements with a memory clobber keep the
        // compiler from forwarding those stores to the later loads (which
        // would hold all sixteen values in registers again).  The item's rows
        // are its own, so no barrier is needed between the two.
        // B200, N = 128, 13,824 of the 54,000 rotations at 512 per
        // launch, with the warp-owned z pass above: 274.3 ms per 54,000
        // rotations against 287.7 for the separate fold pass; holding both
        // row sets in registers spilled and took 298.0.
        auto zpair = [&](float2 &a, float2 &c, int k) {
            const float2 w = conjf2(tw_at(k));
            const float2 w2 = make_float2(-w.x, w.y);
            const float2 e1 = make_float2(a.x + c.x, a.y - c.y), d1 = make_float2(a.x - c.x, a.y + c.y);
            const float2 e2 = make_float2(c.x + a.x, c.y - a.y), d2 = make_float2(c.x - a.x, c.y + a.y);
            const float2 o1 = cmul(w, d1), o2 = cmul(w2, d2);
            a = make_float2(e1.x - o1.y, e1.y + o1.x);
            c = make_float2(e2.x - o2.y, e2.y + o2.x);
        };
        MDB_K3_ITEMS(it, N * (Q2 / 2)) {
            const int z = it % N, g = it / N;
            const int ta = g, tb = g == 0 ? Q2 / 2 : Q2 - g;
            auto row = [&](int r) -> float2 & { return S[r * PITCH + z]; };
            if (g == 0) {
                float2 v[Q1];
                static_for<0, Q1>([&](auto m_) { v[decltype(m_)::value] = row(Q2 * decltype(m_)::value); });
                v[0] = make_float2(v[0].x + v[0].y, v[0].x - v[0].y);
                static_for<1, Q1 / 2 + 1>([&](auto m_) {
                    constexpr int mm = decltype(m_)::value;
                    if constexpr (2 * mm == Q1) {
                        float2 c = v[mm];
                        zpair(v[mm], c, Q2 * mm);
                    } else {
                        zpair(v[mm], v[Q1 - mm], Q2 * mm);
                    }
                });
                static_for<0, Q1>([&](auto m_) { row(Q2 * decltype(m_)::value) = v[decltype(m_)::value]; });
                asm volatile("" ::: "memory");
                static_for<0, Q1>([&](auto m_) { v[decltype(m_)::value] = row(Q2 / 2 + Q2 * decltype(m_)::value); });
                static_for<0, Q1 / 2>([&](auto m_) {
                    constexpr int mm = decltype(m_)::value;
                    zpair(v[mm], v[Q1 - 1 - mm], Q2 / 2 + Q2 * mm);
                });
                static_for<0, Q1>([&](auto m_) { row(Q2 / 2 + Q2 * decltype(m_)::value) = v[decltype(m_)::value]; });
            } else {
                static_for<0, 2>([&](auto h_) {
                    constexpr int h = decltype(h_)::value;
                    float2 a[Q1 / 2], c[Q1 / 2];
                    static_for<0, Q1 / 2>([&](auto j_) {
                        constexpr int j = decltype(j_)::value, mm = h * (Q1 / 2) + j;
                        a[j] = row(ta + Q2 * mm);
                        c[j] = row(tb + Q2 * (Q1 - 1 - mm));
                    });
                    static_for<0, Q1 / 2>([&](auto j_) {
                        constexpr int j = decltype(j_)::value, mm = h * (Q1 / 2) + j;
                        zpair(a[j], c[j], ta + Q2 * mm);
                    });
                    static_for<0, Q1 / 2>([&](auto j_) {
                        constexpr int j = decltype(j_)::value, mm = h * (Q1 / 2) + j;
                        row(ta + Q2 * mm) = a[j];
                        row(tb + Q2 * (Q1 - 1 - mm)) = c[j];
                    });
                    asm volatile("" ::: "memory");
                });
            }
            asm volatile("" ::: "memory");
            static_for<0, 2>([&](auto s_) {
                const int tt = decltype(s_)::value == 0 ? ta : tb;
                float2 v[Q1];
                static_for<0, Q1>([&](auto m_) { v[decltype(m_)::value] = row(tt + Q2 * decltype(m_)::value); });
                Dft<Q1, +1>::run(v);
                static_for<0, Q1>([&](auto k1_) {
                    constexpr int k1 = decltype(k1_)::value;
                    float2 xv = v[k1];
                    if constexpr (k1 != 0) xv = cmul(xv, conjf2(tw_at(2 * tt * k1)));
                    row(k1 * Q2 + tt) = xv;
                });
                asm volatile("" ::: "memory");
            });
        }
    } else {
        // (2a) fold the half spectrum into Z, in place (pairs k, N/2-k)
        MDB_K3_ITEMS(it, N * (NH / 2 + 1)) {
            const int z = it % N, k = it / N;
            if (k == 0) {
                const float2 v = S[z];   // X0 + i X_{N/2}, both real
                S[z] = make_float2(v.x + v.y, v.x - v.y);
            } else {
                const int k2 = NH - k;
                const float2 a = S[k * PITCH + z], c = S[k2 * PITCH + z];
                const float2 wk = conjf2(tw_at(k)), wk2 = conjf2(tw_at(k2));
                // E = a + conj(c), D = a - conj(c), Z = E + i w^k D
                const float2 e1 = make_float2(a.x + c.x, a.y - c.y), d1 = make_float2(a.x - c.x, a.y + c.y);
                const float2 o1 = cmul(wk, d1);
                const float2 z1 = make_float2(e1.x - o1.y, e1.y + o1.x);
                if (k2 != k) {
                    const float2 e2 = make_float2(c.x + a.x, c.y - a.y), d2 = make_float2(c.x - a.x, c.y + a.y);
                    const float2 o2 = cmul(wk2, d2);
                    S[k2 * PITCH + z] = make_float2(e2.x - o2.y, e2.y + o2.x);
                }
                S[k * PITCH + z] = z1;
            }
        }
        __syncthreads();
        // (2b) N/2-point inverse along ky, pass 1 (lanes = z), in place
        MDB_K3_ITEMS(it, N * Q2) {
            const int z = it % N, tt = it / N;
            float2 v[Q1];
            static_for<0, Q1>([&](auto m_) {
                constexpr int mm = decltype(m_)::value;
                v[mm] = S[(tt + Q2 * mm) * PITCH + z];
            });
            Dft<Q1, +1>::run(v);
            static_for<0, Q1>([&](auto k1_) {
                constexpr int k1 = decltype(k1_)::value;
                float2 xv = v[k1];
                if constexpr (k1 != 0) xv = cmul(xv, conjf2(tw_at(2 * tt * k1)));
                S[(k1 * Q2 + tt) * PITCH + z] = xv;
            });
        }
    }
    __syncthreads();
    // (2c) pass 2 -> scores s[2m], s[2m+1] -> per-thread top-T
    TopList<T> top;
    top.init();
    Cand floor{0.f, -1};
    Cand *out = cand + ((size_t)b * N + x) * t + out0;
    if (out0 > 0) {
        floor = out[-1];
        if (floor.idx < 0) {   // an earlier pass already ran out of cells
            if (tid == 0)
                for (int r = 0; r < nsel; ++r) out[r] = Cand{0.f, -1};
            return;
        }
    }
    const int base = x * N * N;
    auto scan = [&](auto floor_on) {
        constexpr bool FL = decltype(floor_on)::value;
        for (int it = tid; it < N * Q1; it += blockDim.x) {
            const int z = it % N, u = it / N;
            float2 o[Q2];
            static_for<0, Q2>([&](auto n2_) {
                constexpr int n2 = decltype(n2_)::value;
                o[n2] = S[(u * Q2 + n2) * PITCH + z];
            });
            Dft<Q2, +1>::run(o);
            const int cell0 = base + 2 * u * N + z;
            static_for<0, Q2>([&](auto k2_) {
                constexpr int k2 = decltype(k2_)::value;
                constexpr int step = 2 * Q1 * k2 * N;   // 2 m2 N - 2 u N for m2 = u + Q1 k2
                top.template insert<FL>(o[k2].x, cell0 + step, floor);
                top.template insert<FL>(o[k2].y, cell0 + step + N, floor);
            });
        }
    };
    if (out0 > 0) {
        // a later pass of T (t > T): the floor from the earlier passes is in
        // force (out0 > 0 with no floor returned above)
        scan(std::true_type{});
    } else {
        // (2c) pass 2: every item keeps only its thread's largest score; the
        // pass's inputs stay in shared memory, so the few threads that pass
        // the bound below recompute their items (the same bits) instead of
        // every thread storing its scores (B200, N = 128: K3 193.4 -> 187.5 ms
        // per 54,000 rotations, identical records).
        float tmax = -INFINITY;   // fmaxf drops NaN keys, which are never selected
        MDB_K3_ITEMS(it, N * Q1) {
            const int z = it % N, u = it / N;
            float2 o[Q2];
            static_for<0, Q2>([&](auto n2_) {
                constexpr int n2 = decltype(n2_)::value;
                o[n2] = S[(u * Q2 + n2) * PITCH + z];
            });
            Dft<Q2, +1>::run(o);
            static_for<0, Q2>([&](auto k2_) {
                constexpr int k2 = decltype(k2_)::value;
                tmax = fmaxf(tmax, fmaxf(o[k2].x, o[k2].y));
            });
        }
        // Threshold: in each warp the nsel-th largest of its lanes' maxima is
        // the key of nsel distinct cells of this plane, so the plane's nsel-th
        // best key is at least that value; the largest such value over the
        // warps bounds it too.  A cell below the bound cannot be among the
        // plane's nsel best, so only cells at or above it enter the lists
        // (equal keys still compete on the index inside the lists).
        __shared__ float thr_w[kNT / 32];
        {
            const int lane = tid & 31, warp = tid >> 5;
            float v = tmax, thw = -INFINITY;
            for (int r = 0; r < nsel; ++r) {
                const int vo = key_ord(v);
                const int mo = __reduce_max_sync(0xffffffffu, vo);
                if (mo == INT_MIN) {   // every lane NaN: no bound from this warp
                    thw = NAN;
                    break;
                }
                thw = ord_key(mo);
                const unsigned holders = __ballot_sync(0xffffffffu, vo == mo);
                if (lane == __ffs(holders) - 1) v = -INFINITY;
            }
            if (lane == 0) thr_w[warp] = thw;
        }
        __syncthreads();
        float thr = thr_w[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) thr = fmaxf(thr, thr_w[w]);
        // the few threads holding a score at or above the bound recompute
        // their items and insert those scores
        if (tmax >= thr) {
            MDB_K3_ITEMS(it, N * Q1) {
                const int z = it % N, u = it / N;
                const int cell0 = base + 2 * u * N + z;
                float2 o[Q2];
                static_for<0, Q2>([&](auto n2_) {
                    constexpr int n2 = decltype(n2_)::value;
                    o[n2] = S[(u * Q2 + n2) * PITCH + z];
                });
                Dft<Q2, +1>::run(o);
                static_for<0, Q2>([&](auto k2_) {
                    constexpr int k2 = decltype(k2_)::value;
                    constexpr int step = 2 * Q1 * k2 * N;
                    const float2 s = o[k2];
                    if (s.x >= thr) top.template insert<false>(s.x, cell0 + step, floor);
                    if (s.y >= thr) top.template insert<false>(s.y, cell0 + step + N, floor);
                });
            }
        }
    }
    // merge: each warp takes its best nsel from its lanes' lists (warp
    // reductions only), then warp 0 takes the plane's best nsel from the
    // warps' lists, with one block barrier in between
    __shared__ Cand wl[kNT / 32][16];
    const int lane = tid & 31, warp = tid >> 5;
    if (__any_sync(0xffffffffu, top.i[0] != INT_MAX)) {
        for (int r = 0; r < nsel; ++r) {
            int owner;
            const Cand c = warp_best(top.head(), owner);
            if (lane == 0) wl[warp][r] = c;
            if (c.idx >= 0 && lane == owner) top.pop();
        }
    } else if (lane < nsel) {
        // no lane of this warp holds a candidate (the common case below the
        // plane's threshold): its list is empty
        wl[warp][lane] = Cand{0.f, -1};
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        int pos = 0;   // this lane's read position in its warp list
        for (int r = 0; r < nsel; ++r) {
            int owner;
            const Cand c = warp_best((lane < nw && pos < nsel) ? wl[lane][pos] : Cand{0.f, -1}, owner);
            if (lane == 0) out[r] = c.idx >= 0 ? c : Cand{0.f, -1};
            if (c.idx < 0) {
                if (lane == 0)
                    for (int r2 = r + 1; r2 < nsel; ++r2) out[r2] = Cand{0.f, -1};
                break;
            }
            if (lane == owner) ++pos;
        }
    }
}

// ------------------------------------------------------------------ K4
// Merge the N x t per-plane candidates of one rotation into t pose records
// with the reference's rules (src/fft_process.cpp:408-458).
static __global__ void k_merge(const Cand *__restrict__ cand, int nplanes, int t, int N, float nf3f, int rot0,
                               DevPose *__restrict__ pose) {
    __shared__ Cand red[33];
    const int b = blockIdx.x;
    const Cand *cb = cand + (size_t)b * nplanes * t;
    const int n = nplanes * t;
    Cand prev{0.f, -1};
    const int N2 = N * N;
    for (int round = 0; round < t; ++round) {
        Cand mine{0.f, -1};
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            const Cand c = cb[e];
            if (c.idx < 0) continue;
            if (prev.idx >= 0 && !key_better(prev.key, prev.idx, c.key, c.idx)) continue;
            if (mine.idx < 0 || key_better(c.key, c.idx, mine.key, mine.idx)) mine = c;
        }
        prev = block_best(mine, red);
        if (threadIdx.x == 0) {
            DevPose r;
            r.rot = rot0 + b;
            int idx = prev.idx;
            float score;
            if (t == 1) {
                // running maximum from 0.0 with strict '<' (src/fft_process.cpp:433-445)
                if (idx < 0 || !(prev.key > 0.f)) {
                    score = 0.f;
                    idx = 0;
                } else {
                    score = __fdiv_rn(prev.key, nf3f);
                }
            } else {
                // insertion below the -99999 sentinel never happens (:408-431)
                score = idx < 0 ? -99999.0f : __fdiv_rn(prev.key, nf3f);
                if (!(score > -99999.0f)) {
                    score = -99999.0f;
                    idx = 0;
                }
            }
            r.score = score;
            r.i = idx / N2;
            r.j = (idx / N) % N;
            r.k = idx % N;
            pose[(size_t)b * t + round] = r;
        }
        if (prev.idx < 0) {
            if (threadIdx.x == 0)
                for (int r2 = round + 1; r2 < t; ++r2)
                    pose[(size_t)b * t + r2] = DevPose{t == 1 ? 0.f : -99999.0f, rot0 + b, 0, 0, 0};
            break;
        }
    }
}

}  // namespace mdb
