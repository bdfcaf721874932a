// md_dock_noalloc: the docking pipeline for callers that cannot allocate
// device memory.
//
// Some callers of a docking library cannot call cudaMalloc: a host framework
// that has already reserved all device memory for its own pool allocator, a
// plugin that must not grow the process's footprint behind its host's back,
// or a latency-critical loop where cudaMalloc/cudaFree (which synchronise the
// device) are not allowed.  This entry point runs the same kernels as md_dock
// but keeps every intermediate in one file-scope static device array, so it
// calls no cudaMalloc, cudaFree or allocating library routine.  The caller
// owns and passes all inputs and outputs as device pointers.
//
// Limits and rules:
//   - scratch is kScratchBytes (32 MiB) per device, held by every device that
//     loads the library until the process exits;
//   - FFT edge nf1 <= 128 (nf1 must have a built kernel set), ligand atoms <=
//     32768, t <= 64, and the per-rotation intermediates must fit the scratch;
//     larger requests return MD_ERR_SIZE;
//   - rotations run one per fused pipeline (the plain form);
//   - the first call on each device does the set-up (symbol address lookup,
//     twiddle tables, kernel attributes) with that device current; make that
//     first call before any stream capture.  Every call looks the scratch
//     address up again (a cheap host query) and repeats the set-up when it
//     changed, as after cudaDeviceReset or in another driver context;
//   - every call shares the one scratch array, which keeps the last call's
//     contents: calls that overlap on the GPU (other streams, other threads)
//     race and must be serialised by the caller.  No scratch region needs
//     clearing: each stage fully overwrites its region before the next reads it.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "../../include/md_b200.h"
#include "dock_kernels.cuh"

using namespace mdb;

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr int kMaxN = 128;
constexpr int kMaxT = 64;
constexpr int kMaxDevices = 64;
// every grid-table size N <= kMaxN
#define MDB_NOALLOC_SIZES(X)                                                                                  \
    X(32) X(36) X(40) X(42) X(44) X(48) X(50) X(54) X(56) X(60) X(64) X(66) X(70) X(72) X(80) X(84) X(88) \
    X(90) X(96) X(98) X(100) X(108) X(110) X(112) X(120) X(126) X(128)
// twiddle tables for every supported N, concatenated
#define MDB_LIST(n) n,
constexpr int kTwSizes[] = {MDB_NOALLOC_SIZES(MDB_LIST)};
#undef MDB_LIST
#define MDB_SUM(n) +n
constexpr int kTwTotal = 0 MDB_NOALLOC_SIZES(MDB_SUM);
#undef MDB_SUM

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];
static __device__ __align__(256) float2 g_twiddle[kTwTotal];

struct DevState {
    bool ready = false;
    unsigned char *scratch = nullptr;
    float2 *twiddle = nullptr;
};
DevState g_state[kMaxDevices];
std::mutex g_mu;

int tw_offset(int n) {
    int off = 0;
    for (int s : kTwSizes) {
        if (s == n) return off;
        off += s;
    }
    return -1;
}

template <int N>
struct Smem {
    static size_t fwd() { return (size_t)N * (N + 1) * sizeof(float2); }
    static size_t xline() { return xline_smem<N, kLT>(); }
    static size_t c2r() { return c2r_smem<N, 0>(); }
};

template <int N>
cudaError_t set_attrs() {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void *f, size_t bytes) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    };
    set((const void *)k_plane_fwd<N, 0>, Smem<N>::fwd());
    set((const void *)k_xline_herm<N, kLT>, Smem<N>::xline());
    set((const void *)k_plane_c2r<N, 1>, Smem<N>::c2r());
    set((const void *)k_plane_c2r<N, 4>, Smem<N>::c2r());
    set((const void *)k_plane_c2r<N, 16>, Smem<N>::c2r());
    return e;
}

// With the device current: the set-up, done again whenever the scratch
// array's address differs from the one the set-up used (a reset device or a
// different driver context loads the module's arrays anew).
int setup(int dev) {
    std::lock_guard<std::mutex> lk(g_mu);
    DevState &st = g_state[dev];
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess) return MD_ERR_CUDA;
    if (st.ready && st.scratch == p) return MD_OK;
    st.ready = false;
    st.scratch = static_cast<unsigned char *>(p);
    if (cudaGetSymbolAddress(&p, g_twiddle) != cudaSuccess) return MD_ERR_CUDA;
    st.twiddle = static_cast<float2 *>(p);
    std::vector<float2> tw;
    tw.reserve(kTwTotal);
    for (int n : kTwSizes)
        for (int j = 0; j < n; ++j) {
            const double a = -2.0 * M_PI * (double)j / (double)n;
            tw.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
        }
    if (cudaMemcpyToSymbol(g_twiddle, tw.data(), sizeof(float2) * kTwTotal) != cudaSuccess) return MD_ERR_CUDA;
    cudaError_t e = cudaSuccess;
#define X(n) \
    if (e == cudaSuccess) e = set_attrs<n>();
    MDB_NOALLOC_SIZES(X)
#undef X
    if (e != cudaSuccess) return MD_ERR_CUDA;
    st.ready = true;
    return MD_OK;
}

__global__ void k_pack_ligand(int na, const float *__restrict__ xyz, const float *__restrict__ radius,
                              const float *__restrict__ charge, float4 *__restrict__ atom, float2 *__restrict__ rad2) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= na) return;
    atom[l] = make_float4(xyz[3 * l], xyz[3 * l + 1], xyz[3 * l + 2], charge[l]);
    // R*R*1.5 and R*R*1.0 in float, as Ligand::precalc (src/ligand.cpp:251-254)
    const float r = radius[l];
    rad2[l] = make_float2(__fmul_rn(__fmul_rn(r, r), 1.5f), __fmul_rn(__fmul_rn(r, r), 1.0f));
}

struct Prep {
    MarkEntry *srec;
    int *sstart;
    int2 *cq;
    int *cstart;
};

template <int N>
void run_rotation(cudaStream_t s, const LigandView &L, const GridView &G, const float *rot9, const float2 *Rh,
                  const Prep &pr, uint32_t *vbits, int2 *qlist, int *qcount, float2 *A, float2 *Gsp, Cand *cand,
                  int rot, int t, DevPose *pose) {
    constexpr int NG = N / 2, NH = N / 2, TILES = (N + kLT - 1) / kLT;
    const float nf3f = (float)((long long)N * N * N);
    k_atom_prep<NG><<<1, kNTP, 0, s>>>(L, G, rot9, pr.srec, pr.sstart, pr.cq, pr.cstart);
    k_vox_bits<NG><<<dim3(NG, 1), kNT0, vox_bits_smem<NG>(), s>>>(L, G, pr.srec, pr.sstart, pr.cq, pr.cstart, vbits,
                                                                 qlist, qcount);
    k_plane_fwd<N, 0><<<dim3(NG, 1), kNT1, Smem<N>::fwd(), s>>>(L, G, vbits, qlist, qcount, nullptr, nullptr, A,
                                                               nullptr, nullptr);
    k_xline_herm<N, kLT><<<dim3(NH * TILES, 1), 16 * kLT, Smem<N>::xline(), s>>>(G, A, Rh, Gsp);
    const int T = t == 1 ? 1 : (t <= 4 ? 4 : 16);
    for (int out0 = 0; out0 < t; out0 += T) {
        const int nsel = t - out0 < T ? t - out0 : T;
        if (T == 1)
            k_plane_c2r<N, 1><<<dim3(N, 1), kNT, Smem<N>::c2r(), s>>>(G, Gsp, t, nf3f, out0, nsel, cand);
        else if (T == 4)
            k_plane_c2r<N, 4><<<dim3(N, 1), kNT, Smem<N>::c2r(), s>>>(G, Gsp, t, nf3f, out0, nsel, cand);
        else
            k_plane_c2r<N, 16><<<dim3(N, 1), kNT, Smem<N>::c2r(), s>>>(G, Gsp, t, nf3f, out0, nsel, cand);
    }
    k_merge<<<1, 256, 0, s>>>(cand, N, t, N, nf3f, rot, pose);
}

}  // namespace

extern "C" int md_dock_noalloc(int nf1, float grid_width, const float *d_grid_coord, const float *d_receptor_spectrum,
                               int na, const float *d_xyz_centred, const float *d_radius, const float *d_charge,
                               float lig_core, const float *d_rotmat, int first_rot, int n_rot, int t,
                               md_pose *d_out, void *stream) {
    if (!d_grid_coord || !d_receptor_spectrum || !d_xyz_centred || !d_radius || !d_charge || !d_rotmat || !d_out)
        return MD_ERR_ARG;
    if (n_rot < 0 || t < 1 || na < 1 || !(grid_width > 0.f)) return MD_ERR_ARG;
    if (lig_core == 0.0f || lig_core == -8888.0f) return MD_ERR_ARG;
    if (nf1 > kMaxN || tw_offset(nf1) < 0 || t > kMaxT || na > kMaxLigAtoms) return MD_ERR_SIZE;
    const size_t N = nf1, NG = nf1 / 2;
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t b_atom = up(sizeof(float4) * na), b_rad = up(sizeof(float2) * na);
    const size_t b_A = up(sizeof(float2) * NG * N * N), b_G = up(sizeof(float2) * N * (N / 2) * N);
    const size_t b_cand = up(sizeof(Cand) * N * t);
    const size_t b_bits = up(sizeof(uint32_t) * NG * 2 * NG * ((NG + 31) / 32));
    const size_t b_ql = up(sizeof(int2) * NG * NG * NG), b_qc = up(sizeof(int) * NG);
    const size_t b_sr = up(sizeof(MarkEntry) * na), b_ss = up(sizeof(int) * (NG + 2 * kReach + 1));
    const size_t b_cq = up(sizeof(int2) * na), b_cs = up(sizeof(int) * (NG + 1));
    const size_t used = b_atom + b_rad + b_A + b_G + b_cand + b_bits + b_ql + b_qc + b_sr + b_ss + b_cq + b_cs;
    if (used > kScratchBytes) return MD_ERR_SIZE;
    if (n_rot == 0) return MD_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MD_ERR_CUDA;
    int rc = setup(dev);
    if (rc) return rc;
    const DevState &st = g_state[dev];
    unsigned char *p = st.scratch;
    float4 *atom = reinterpret_cast<float4 *>(p);
    float2 *rad2 = reinterpret_cast<float2 *>(p + b_atom);
    float2 *A = reinterpret_cast<float2 *>(p + b_atom + b_rad);
    float2 *Gsp = reinterpret_cast<float2 *>(p + b_atom + b_rad + b_A);
    Cand *cand = reinterpret_cast<Cand *>(p + b_atom + b_rad + b_A + b_G);
    uint32_t *vbits = reinterpret_cast<uint32_t *>(p + b_atom + b_rad + b_A + b_G + b_cand);
    int2 *qlist = reinterpret_cast<int2 *>(p + b_atom + b_rad + b_A + b_G + b_cand + b_bits);
    int *qcount = reinterpret_cast<int *>(p + b_atom + b_rad + b_A + b_G + b_cand + b_bits + b_ql);
    unsigned char *q0 = p + b_atom + b_rad + b_A + b_G + b_cand + b_bits + b_ql + b_qc;
    const Prep prep{reinterpret_cast<MarkEntry *>(q0), reinterpret_cast<int *>(q0 + b_sr),
                    reinterpret_cast<int2 *>(q0 + b_sr + b_ss), reinterpret_cast<int *>(q0 + b_sr + b_ss + b_cq)};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_pack_ligand<<<(na + 255) / 256, 256, 0, s>>>(na, d_xyz_centred, d_radius, d_charge, atom, rad2);
    GridView G{(int)NG, grid_width, (float)((int)NG * grid_width) / 2, d_grid_coord, st.twiddle + tw_offset(nf1)};
    LigandView L{na, atom, rad2, lig_core};
    const float2 *Rh = reinterpret_cast<const float2 *>(d_receptor_spectrum);
    DevPose *pose = reinterpret_cast<DevPose *>(d_out);
    for (int r = 0; r < n_rot; ++r) {
        const float *rot9 = d_rotmat + 9 * (size_t)r;
        DevPose *pr = pose + (size_t)r * t;
        switch (nf1) {
#define X(n) \
    case n: run_rotation<n>(s, L, G, rot9, Rh, prep, vbits, qlist, qcount, A, Gsp, cand, first_rot + r, t, pr); break;
            MDB_NOALLOC_SIZES(X)
#undef X
        }
    }
    return cudaGetLastError() == cudaSuccess ? MD_OK : MD_ERR_CUDA;
}
