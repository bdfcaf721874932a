// Device context shared by the C-ABI translation units: the per-launch work
// sets, the context struct and the per-size pipeline (Sized<N>).  Each FFT
// size's kernels are instantiated in one of the sized_*.cu files, which
// export a SizedOps table; md_b200.cu dispatches through it, so the sizes
// compile in parallel.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/md_b200.h"
#include "dock_kernels.cuh"
#include "staged_kernels.cuh"

using namespace mdb;

namespace mdb {

// Candidate groups per rotation from the top-t kernels: one per x-plane, or
// one per (x-plane, column block) for the staged sizes.
inline size_t cand_groups(size_t N) {
    return N > (size_t)kMaxResidentN ? N * ((N + kCB - 1) / kCB) : N;
}

// Per-launch intermediates for `cap` rotations of one launch group.
struct WorkSet {
    float2 *A = nullptr;        // [cap][N/2][N][N]    spectrum planes (K1 -> K2)
    float2 *G = nullptr;        // [cap][N][N/2][N]    Hermitian half (K2 -> K3)
    Cand *cand = nullptr;       // [cap][groups][t]    per-plane candidates (K3 -> K4)
    uint32_t *vbits = nullptr;  // [cap][N/2][2][N/2 * words per row] voxel classes (K0 -> K1)
    int2 *qlist = nullptr;      // [cap][N/2][(N/2)^2] charged cells per voxel plane (K0 -> K1)
    int *qcount = nullptr;      // [cap][N/2]
    MarkEntry *srec = nullptr;  // [cap][na]           atom records bucketed by plane (prep -> K0)
    int *sstart = nullptr;      // [cap][N/2 + 2 kReach + 1]
    int2 *cq = nullptr;         // [cap][na]           charge entries bucketed by plane, atom order
    int *cstart = nullptr;      // [cap][N/2 + 1]
    uint32_t *marks = nullptr;  // [cap][N/2][2][N/2 * words per row] core / surface marks (K0m -> K0)

    void release() {
        cudaFree(A);
        cudaFree(G);
        cudaFree(cand);
        cudaFree(vbits);
        cudaFree(qlist);
        cudaFree(qcount);
        cudaFree(srec);
        cudaFree(sstart);
        cudaFree(cq);
        cudaFree(cstart);
        cudaFree(marks);
        *this = WorkSet();
    }
    // Bytes of each buffer for launch groups of `cap` rotations.
    static constexpr int kBufs = 11;
    struct Sizes {
        size_t b[kBufs];
    };
    static Sizes need(size_t cap, size_t N, size_t t, size_t na) {
        const size_t NG = N / 2;
        return Sizes{{sizeof(float2) * cap * NG * N * N, sizeof(float2) * cap * N * (N / 2) * N,
                      sizeof(Cand) * cap * cand_groups(N) * t, sizeof(uint32_t) * cap * NG * 2 * NG * ((NG + 31) / 32),
                      sizeof(int2) * cap * NG * NG * NG, sizeof(int) * cap * NG, sizeof(MarkEntry) * cap * na,
                      sizeof(int) * cap * (NG + 2 * kReach + 1), sizeof(int2) * cap * na, sizeof(int) * cap * (NG + 1),
                      sizeof(uint32_t) * cap * NG * 2 * NG * ((NG + 31) / 32)}};
    }
    cudaError_t allocate(const Sizes &z) {
        cudaError_t e = cudaSuccess;
        void **slot[kBufs] = {(void **)&A,    (void **)&G,    (void **)&cand,   (void **)&vbits,
                              (void **)&qlist, (void **)&qcount, (void **)&srec, (void **)&sstart,
                              (void **)&cq,   (void **)&cstart, (void **)&marks};
        for (int k = 0; k < kBufs && e == cudaSuccess; ++k) e = cudaMalloc(slot[k], z.b[k]);
        return e;
    }
};

constexpr int kLanes = 2;

}  // namespace

struct md_ctx {
    int device = 0;
    // Identity of this context's captured state for other contexts' graph
    // caches: uid is never reused within the process (a later context at the
    // same heap address gets a new one) and gen is bumped whenever a change
    // invalidates this context's own captured graphs (free_graphs).
    uint64_t uid = 0;
    uint64_t gen = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;     // second capture stream of the batched form
    cudaEvent_t fork = nullptr, join = nullptr;
    std::string err;
    // grid
    int N = 0, ng = 0;
    float gw = 0.f;
    float *d_gc = nullptr;
    float2 *d_tw = nullptr;
    // receptor spectrum [kx][ky][kz] and the receptor voxel grids (for the adjoint)
    float2 *d_Rh = nullptr;
    float *d_recv = nullptr;   // [2][ng^3] real, imaginary
    bool have_receptor = false;
    // ligand
    int na = 0, na_cap = 0;
    float delta = 1.0f;
    float4 *d_atom = nullptr;
    float2 *d_rad2 = nullptr;
    bool have_ligand = false;
    // work sets (lane 0 serves every form; lane 1 the batched graph)
    int batch = 1;
    int plan = 0;   // radix plan variant of the plane top-t kernel (C2RPlan)
    int tile = 32;  // kz lines per CTA of the x-line kernel (8, 16 or 32)
    int lanes = kLanes;   // work sets / capture streams the batched graph alternates over (1 or 2)
    int cap = 0, cap_t = 0, cap_na = 0;
    WorkSet::Sizes have{};           // bytes held by each work-set buffer
    int sets = 0;                    // work sets allocated (1 or kLanes)
    WorkSet ws[kLanes];
    char *d_scratch = nullptr;   // scratch of the adjoint and pose-scoring calls (grows to the largest call)
    size_t scratch_cap = 0;
    // staging for host-buffer calls
    float *d_rot = nullptr;
    size_t rot_cap = 0;
    DevPose *d_pose = nullptr;
    size_t pose_cap = 0;
    // captured graphs of the batched form: (first_rot, n_rot, t, batch, rot ptr, pose ptr)
    std::map<std::tuple<int, int, int, int, const float *, DevPose *>, cudaGraphExec_t> graphs;
    // captured graphs of md_dock_pairs, keyed by every argument
    std::map<std::vector<uintptr_t>, cudaGraphExec_t> pair_graphs;
};

static_assert(sizeof(md_pose) == sizeof(DevPose), "pose layout");

#define MD_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                     \
            return MD_ERR_CUDA;                                                                \
        }                                                                                      \
    } while (0)

namespace mdb {

// ------------------------------------------------------------------ per-size dispatch
template <int N>
struct Sized {
    static constexpr int NG = N / 2;
    static constexpr int NH = N / 2;
    static constexpr int TILES = (N + kLT - 1) / kLT;
    // above 224 the plane transforms run as row and column launches
    // (staged_kernels.cuh)
    static constexpr bool kStaged = staged<N>();
    static constexpr int ZB = c2r_zblocks<N>();
    static size_t smem_fwd() { return (size_t)N * (N + 1) * sizeof(float2); }
    static size_t smem_xrec() { return (size_t)N * kLT * sizeof(float2); }
    static size_t smem_vox() { return vox_bits_smem<NG>(); }
    // the column-block forward form: always for MODE 0 where two CTAs fit, and
    // for every mode where the one-CTA plane does not fit
    template <int MODE>
    static constexpr bool use_cb() {
        return !fwd_full_fits<N>() || (MODE == 0 && fwd_cb_fits<N>());
    }
    template <int MODE, class Set>
    static void set_fwd(Set &set) {
        if constexpr (use_cb<MODE>()) set((const void *)k_plane_fwd_cb<N, MODE>, fwd_cb_smem<N>());
        else set((const void *)k_plane_fwd<N, MODE>, smem_fwd());
    }
    template <int MODE>
    static void plane_fwd(cudaStream_t s, int nb, const LigandView &L, const GridView &G, const uint32_t *vbits,
                          const int2 *qlist, const int *qcount, const float *sr, const float *si, float2 *A,
                          float *vr, float *vi) {
        if constexpr (use_cb<MODE>())
            k_plane_fwd_cb<N, MODE><<<dim3(NG, nb), kNT1B, fwd_cb_smem<N>(), s>>>(L, G, vbits, qlist, qcount, sr, si,
                                                                                   A, vr, vi);
        else
            k_plane_fwd<N, MODE><<<dim3(NG, nb), kNT1, smem_fwd(), s>>>(L, G, vbits, qlist, qcount, sr, si, A, vr, vi);
    }
    template <int LT = kLT>
    static size_t smem_xline() { return xline_smem<N, LT>(); }
    template <int V = 0>
    static size_t smem_c2r() { return c2r_smem<N, V>(); }

    static cudaError_t set_attrs() {
        static bool done = false;
        if (done) return cudaSuccess;
        cudaError_t e = cudaSuccess;
        auto set = [&](const void *f, size_t bytes) {
            if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        };
        if constexpr (kStaged) {
            set((const void *)k_rows_fwd<N, 0>, rows_smem(N));
            set((const void *)k_rows_fwd<N, 1>, rows_smem(N));
            set((const void *)k_rows_fwd<N, 2>, rows_smem(N));
            set((const void *)k_cols_fwd<N>, cols_fwd_smem(N));
            set((const void *)k_rows_inv<N>, rows_smem(N));
            set((const void *)k_cols_c2r<N, 1>, cols_c2r_smem(N));
            set((const void *)k_cols_c2r<N, 4>, cols_c2r_smem(N));
            set((const void *)k_cols_c2r<N, 16>, cols_c2r_smem(N));
        } else {
            set_fwd<0>(set);
            set_fwd<1>(set);
            set_fwd<2>(set);
            set((const void *)k_plane_c2r<N, 1, 0>, smem_c2r<0>());
            set((const void *)k_plane_c2r<N, 4, 0>, smem_c2r<0>());
            set((const void *)k_plane_c2r<N, 16, 0>, smem_c2r<0>());
            set((const void *)k_plane_c2r<N, 1, 1>, smem_c2r<1>());
            set((const void *)k_plane_c2r<N, 4, 1>, smem_c2r<1>());
            set((const void *)k_plane_c2r<N, 1, 2>, smem_c2r<2>());
            set((const void *)k_plane_c2r<N, 4, 2>, smem_c2r<2>());
        }
        set((const void *)k_xline_rec<N>, smem_xrec());
        set((const void *)k_vox_bits<NG, true>, smem_vox());
        set((const void *)k_vox_bits<NG, false>, smem_vox());
        if constexpr (xline_tile_fits<N, 32>()) set((const void *)k_xline_herm<N, 32>, smem_xline<32>());
        set((const void *)k_xline_herm<N, 16>, smem_xline<16>());
        set((const void *)k_xline_herm<N, 8>, smem_xline<8>());
        if constexpr (xline_fold_ok<N>()) set((const void *)k_xline_fold<N, 16>, smem_xline<16>());
        if (e == cudaSuccess) done = true;
        return e;
    }

    // Forward plane transforms of nb rotations (MODE 0/1) or the voxel planes
    // themselves (MODE 2) in the staged form: row launch, then column launch.
    template <int MODE>
    static void staged_fwd(cudaStream_t s, int nb, const LigandView &L, const GridView &G, const uint32_t *vbits,
                           const int2 *qlist, const int *qcount, const float *sr, const float *si, float2 *A,
                           float *vr, float *vi) {
        k_rows_fwd<N, MODE><<<dim3(NG, (NG + kRB - 1) / kRB, nb), kNTS, rows_smem(N), s>>>(L, G, vbits, qlist, qcount,
                                                                                           sr, si, A, vr, vi);
        if constexpr (MODE != 2) k_cols_fwd<N><<<dim3(NG, (N + kCB - 1) / kCB, nb), kNTS, cols_fwd_smem(N), s>>>(G, A);
    }
    template <int MODE>
    static void any_fwd(cudaStream_t s, int nb, const LigandView &L, const GridView &G, const uint32_t *vbits,
                        const int2 *qlist, const int *qcount, const float *sr, const float *si, float2 *A, float *vr,
                        float *vi) {
        if constexpr (kStaged) staged_fwd<MODE>(s, nb, L, G, vbits, qlist, qcount, sr, si, A, vr, vi);
        else plane_fwd<MODE>(s, nb, L, G, vbits, qlist, qcount, sr, si, A, vr, vi);
    }

    static void receptor(md_ctx *c, const float *d_r, const float *d_i) {
        GridView G{c->ng, c->gw, 0.f, c->d_gc, c->d_tw};
        LigandView L{0, nullptr, nullptr, 1.f};
        any_fwd<1>(c->stream, 1, L, G, nullptr, nullptr, nullptr, d_r, d_i, c->ws[0].A, nullptr, nullptr);
        k_xline_rec<N><<<dim3(N * TILES, 1), kNT, smem_xrec(), c->stream>>>(G, c->ws[0].A, c->d_Rh);
    }

    // Voxelizer of one launch group (atom prep + K0).
    static void voxelize(md_ctx *c, const WorkSet &w, const float *d_rot9, int nb, cudaStream_t s) {
        GridView G{c->ng, c->gw, (float)(c->ng * c->gw) / 2, c->d_gc, c->d_tw};
        LigandView L{c->na, c->d_atom, c->d_rad2, c->delta};
        k_atom_prep<NG><<<nb, kNTP, 0, s>>>(L, G, d_rot9, w.srec, w.sstart, w.cq, w.cstart);
        k_vox_mark<NG><<<dim3(NG, nb), kNT0, 0, s>>>(L, G, w.srec, w.sstart, w.marks);
        k_vox_bits<NG, true><<<dim3(NG, nb), kNT0, smem_vox(), s>>>(L, G, w.srec, w.sstart, w.cq, w.cstart,
                                                                   w.vbits, w.qlist, w.qcount, w.marks);
    }

    // Voxel grids of nb rotations ([nb][ng^3] real, imaginary) into vr / vi.
    static void voxel_chunk(md_ctx *c, const float *d_rot9, int nb, float *d_vr, float *d_vi) {
        GridView G{c->ng, c->gw, (float)(c->ng * c->gw) / 2, c->d_gc, c->d_tw};
        LigandView L{c->na, c->d_atom, c->d_rad2, c->delta};
        const WorkSet &w = c->ws[0];
        voxelize(c, w, d_rot9, nb, c->stream);
        any_fwd<2>(c->stream, nb, L, G, w.vbits, w.qlist, w.qcount, nullptr, nullptr, nullptr, d_vr, d_vi);
    }

    static void voxels(md_ctx *c, const float *d_rot9, float *d_vr, float *d_vi) {
        GridView G{c->ng, c->gw, (float)(c->ng * c->gw) / 2, c->d_gc, c->d_tw};
        LigandView L{c->na, c->d_atom, c->d_rad2, c->delta};
        const WorkSet &w = c->ws[0];
        voxelize(c, w, d_rot9, 1, c->stream);
        any_fwd<2>(c->stream, 1, L, G, w.vbits, w.qlist, w.qcount, nullptr, nullptr, nullptr, d_vr, d_vi);
    }

    // The plane top-t kernel in passes of T candidates (T = 1, 4 or 16), with
    // radix plan variant `plan` (T = 16 always uses variant 0).
    template <int T, int V>
    static void c2r(cudaStream_t s, const GridView &G, const float2 *Gh, int nb, int t, float nf3f, int out0,
                    int nsel, Cand *cand) {
        k_plane_c2r<N, T, V><<<dim3(N, nb), kNT, smem_c2r<V>(), s>>>(G, Gh, t, nf3f, out0, nsel, cand);
    }
    static void plane_topt(cudaStream_t s, const GridView &G, float2 *Gh, int nb, int t, float nf3f, Cand *cand,
                           int plan) {
        const int T = t == 1 ? 1 : (t <= 4 ? 4 : 16);
        if constexpr (kStaged) {
            k_rows_inv<N><<<dim3(N, (NH + kRB - 1) / kRB, nb), kNTS, rows_smem(N), s>>>(G, Gh);
            for (int out0 = 0; out0 < t; out0 += T) {
                const int nsel = std::min(T, t - out0);
                const dim3 grid(N, ZB, nb);
                if (T == 1) k_cols_c2r<N, 1><<<grid, kNTS, cols_c2r_smem(N), s>>>(G, Gh, t, out0, nsel, cand);
                else if (T == 4) k_cols_c2r<N, 4><<<grid, kNTS, cols_c2r_smem(N), s>>>(G, Gh, t, out0, nsel, cand);
                else k_cols_c2r<N, 16><<<grid, kNTS, cols_c2r_smem(N), s>>>(G, Gh, t, out0, nsel, cand);
            }
        } else {
            for (int out0 = 0; out0 < t; out0 += T) {
                const int nsel = std::min(T, t - out0);
                if (T == 1) {
                    if (plan == 1) c2r<1, 1>(s, G, Gh, nb, t, nf3f, out0, nsel, cand);
                    else if (plan == 2) c2r<1, 2>(s, G, Gh, nb, t, nf3f, out0, nsel, cand);
                    else c2r<1, 0>(s, G, Gh, nb, t, nf3f, out0, nsel, cand);
                } else if (T == 4) {
                    if (plan == 1) c2r<4, 1>(s, G, Gh, nb, t, nf3f, out0, nsel, cand);
                    else if (plan == 2) c2r<4, 2>(s, G, Gh, nb, t, nf3f, out0, nsel, cand);
                    else c2r<4, 0>(s, G, Gh, nb, t, nf3f, out0, nsel, cand);
                } else {
                    c2r<16, 0>(s, G, Gh, nb, t, nf3f, out0, nsel, cand);
                }
            }
        }
    }

    // One launch group: nb rotations whose matrices start at d_rot9, on work
    // set w and stream s.  With `ev` set, an event is recorded after each of
    // the five stages.
    static void dock(md_ctx *c, const WorkSet &w, cudaStream_t s, const float *d_rot9, int nb, int rot0, int t,
                     DevPose *d_pose, cudaEvent_t *ev) {
        GridView G{c->ng, c->gw, (float)(c->ng * c->gw) / 2, c->d_gc, c->d_tw};
        LigandView L{c->na, c->d_atom, c->d_rad2, c->delta};
        const float nf3f = (float)((long long)N * N * N);
        voxelize(c, w, d_rot9, nb, s);
        if (ev) cudaEventRecord(ev[1], s);
        any_fwd<0>(s, nb, L, G, w.vbits, w.qlist, w.qcount, nullptr, nullptr, w.A, nullptr, nullptr);
        if (ev) cudaEventRecord(ev[2], s);
        bool folded = false;   // the register-fold form, instantiated only where it is used
        if constexpr (xline_fold_ok<N>()) {
            if (c->tile == 16) {
                k_xline_fold<N, 16><<<xline_grid<N>(NH * ((N + 15) / 16), nb), 256, smem_xline<16>(), s>>>(
                    G, w.A, c->d_Rh, w.G);
                folded = true;
            }
        }
        if (folded) {
        } else if (c->tile == 16)
            k_xline_herm<N, 16><<<xline_grid<N>(NH * ((N + 15) / 16), nb), 256, smem_xline<16>(), s>>>(G, w.A, c->d_Rh,
                                                                                                      w.G);
        else if (c->tile == 8)
            k_xline_herm<N, 8><<<xline_grid<N>(NH * ((N + 7) / 8), nb), 128, smem_xline<8>(), s>>>(G, w.A, c->d_Rh, w.G);
        else if constexpr (xline_tile_fits<N, 32>())
            k_xline_herm<N, 32><<<xline_grid<N>(NH * ((N + 31) / 32), nb), 512, smem_xline<32>(), s>>>(G, w.A, c->d_Rh,
                                                                                                      w.G);
        else
            k_xline_herm<N, 16><<<xline_grid<N>(NH * ((N + 15) / 16), nb), 256, smem_xline<16>(), s>>>(G, w.A, c->d_Rh,
                                                                                                      w.G);
        if (ev) cudaEventRecord(ev[3], s);
        plane_topt(s, G, w.G, nb, t, nf3f, w.cand, c->plan);
        if (ev) cudaEventRecord(ev[4], s);
        k_merge<<<nb, 256, 0, s>>>(w.cand, kStaged ? N * ZB : N, t, N, nf3f, rot0, d_pose);
        if (ev) cudaEventRecord(ev[5], s);
    }
};

}  // namespace mdb

namespace mdb {

// The per-size pipeline entry points of one FFT size.
struct SizedOps {
    int N;
    cudaError_t (*set_attrs)();
    void (*receptor)(md_ctx *, const float *, const float *);
    void (*voxel_chunk)(md_ctx *, const float *, int, float *, float *);
    void (*voxels)(md_ctx *, const float *, float *, float *);
    void (*dock)(md_ctx *, const WorkSet &, cudaStream_t, const float *, int, int, int, DevPose *, cudaEvent_t *);
};

template <int N>
const SizedOps *sized_ops_of() {
    static const SizedOps ops{N, &Sized<N>::set_attrs, &Sized<N>::receptor, &Sized<N>::voxel_chunk,
                              &Sized<N>::voxels, &Sized<N>::dock};
    return &ops;
}

// Defined by the sized_*.cu files: the table of N, or nullptr.
const SizedOps *sized_ops_a(int N);
const SizedOps *sized_ops_b(int N);
const SizedOps *sized_ops_c(int N);
const SizedOps *sized_ops_d(int N);
const SizedOps *sized_ops_e(int N);
const SizedOps *sized_ops_f(int N);
const SizedOps *sized_ops_g(int N);
const SizedOps *sized_ops_h(int N);
const SizedOps *sized_ops_i(int N);
const SizedOps *sized_ops_j(int N);
const SizedOps *sized_ops_k(int N);
const SizedOps *sized_ops_l(int N);
const SizedOps *sized_ops_m(int N);
const SizedOps *sized_ops_n(int N);
const SizedOps *sized_ops_o(int N);
const SizedOps *sized_ops_p(int N);
const SizedOps *sized_ops_q(int N);
const SizedOps *sized_ops_r(int N);

inline const SizedOps *sized_ops(int N) {
    if (const SizedOps *o = sized_ops_a(N)) return o;
    if (const SizedOps *o = sized_ops_b(N)) return o;
    if (const SizedOps *o = sized_ops_c(N)) return o;
    if (const SizedOps *o = sized_ops_d(N)) return o;
    if (const SizedOps *o = sized_ops_e(N)) return o;
    if (const SizedOps *o = sized_ops_f(N)) return o;
    if (const SizedOps *o = sized_ops_g(N)) return o;
    if (const SizedOps *o = sized_ops_h(N)) return o;
    if (const SizedOps *o = sized_ops_i(N)) return o;
    if (const SizedOps *o = sized_ops_j(N)) return o;
    if (const SizedOps *o = sized_ops_k(N)) return o;
    if (const SizedOps *o = sized_ops_l(N)) return o;
    if (const SizedOps *o = sized_ops_m(N)) return o;
    if (const SizedOps *o = sized_ops_n(N)) return o;
    if (const SizedOps *o = sized_ops_o(N)) return o;
    if (const SizedOps *o = sized_ops_p(N)) return o;
    if (const SizedOps *o = sized_ops_q(N)) return o;
    return sized_ops_r(N);
}

}  // namespace mdb
