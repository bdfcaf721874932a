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
#include "fft_dev.cuh"

namespace mdb {

constexpr int kNT = 512;          // threads per CTA for the plane kernels
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

// Mark core / surface bits of planes around p for every atom near p.
template <int NG>
__device__ void vox_mark(VoxShared<NG> &vs, const LigandView &L, const GridView &G, const float *m, int p,
                         bool general_delta) {
    constexpr int W = VoxShared<NG>::W;
    const int ng = G.ng;
    const int reach = general_delta ? 4 : 3;
    const int plo = general_delta ? -2 : -1, phi = general_delta ? 2 : 1;
    for (int l = threadIdx.x; l < L.na; l += blockDim.x) {
        const float4 a = __ldg(&L.atom[l]);
        const float xr = rot_x(m, a.x, a.y, a.z);
        const int i2 = box_origin(xr, G.gw, ng);
        if (i2 < p - reach || i2 > p + reach) continue;
        const float yr = rot_x(m + 3, a.x, a.y, a.z);
        const float zr = rot_x(m + 6, a.x, a.y, a.z);
        const int j2 = box_origin(yr, G.gw, ng);
        const int k2 = box_origin(zr, G.gw, ng);
        const float2 r2 = __ldg(&L.rad2[l]);
        const int ia = max(i2 - 2, max(0, p + plo)), ib = min(i2 + 3, min(ng, p + phi + 1));
        const int ja = max(j2 - 2, 0), jb = min(j2 + 3, ng);
        const int ka = max(k2 - 2, 0), kb = min(k2 + 3, ng);
        for (int i = ia; i < ib; ++i) {
            const float xd = sqdist(xr, __ldg(&G.gc[i]));
            const int slot = i - p + 2;
            const bool do_surf = (i >= p - 1 && i <= p + 1);
            for (int j = ja; j < jb; ++j) {
                const float d2 = __fadd_rn(xd, sqdist(yr, __ldg(&G.gc[j])));
                uint32_t cbits[W], sbits[W];
#pragma unroll
                for (int w = 0; w < W; ++w) cbits[w] = sbits[w] = 0u;
                for (int k = ka; k < kb; ++k) {
                    const float d3 = __fadd_rn(d2, sqdist(zr, __ldg(&G.gc[k])));
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        if ((k >> 5) == w) {
                            if (d3 < r2.x) cbits[w] |= 1u << (k & 31);
                            if (d3 < r2.y) sbits[w] |= 1u << (k & 31);
                        }
                    }
                }
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    if (cbits[w]) atomicOr(&vs.core[slot][j * W + w], cbits[w]);
                    if (do_surf && sbits[w]) atomicOr(&vs.surf[slot - 1][j * W + w], sbits[w]);
                }
            }
        }
    }
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

// Real rPSC value of cell (p, q, s).
template <int NG>
__device__ __forceinline__ float vox_real(const VoxShared<NG> &vs, int p, int q, int s, int ng, float delta,
                                          bool general_delta) {
    const int c = vox_class<NG>(vs, 2, p, q, s, ng);
    if (c == 1) return 1.0f;
    if (c == 0) return 0.0f;
    if (general_delta) {
        // src/ligand.cpp:176-195: interior core cells next to an empty cell -> 1.0
        const bool interior = p >= 1 && p <= ng - 2 && q >= 1 && q <= ng - 2 && s >= 1 && s <= ng - 2;
        if (interior) {
            if (vox_class<NG>(vs, 1, p - 1, q, s, ng) == 0 || vox_class<NG>(vs, 3, p + 1, q, s, ng) == 0 ||
                vox_class<NG>(vs, 2, p, q - 1, s, ng) == 0 || vox_class<NG>(vs, 2, p, q + 1, s, ng) == 0 ||
                vox_class<NG>(vs, 2, p, q, s - 1, ng) == 0 || vox_class<NG>(vs, 2, p, q, s + 1, ng) == 0)
                return 1.0f;
        }
    }
    return delta;
}

// Charges of the atoms whose charge cell lies in plane p, added per cell in
// ascending atom order starting from the cell's current value, exactly as the
// sequential loop of src/ligand.cpp:216-234 rounds them.  `flags` is a bitmap
// over atoms in shared memory; `cell(q, s)` returns a reference to the
// cell's imaginary part.
template <class Cell>
__device__ void vox_charges(uint32_t *flags, const LigandView &L, const GridView &G, const float *m, int p,
                            Cell cell) {
    const int nw = (L.na + 31) >> 5;
    for (int w = threadIdx.x; w < nw; w += blockDim.x) flags[w] = 0u;
    __syncthreads();
    for (int l = threadIdx.x; l < L.na; l += blockDim.x) {
        const float4 a = __ldg(&L.atom[l]);
        const float xr = rot_x(m, a.x, a.y, a.z);
        if (charge_cell(xr, G.pad, G.gw, G.ng) == p) atomicOr(&flags[l >> 5], 1u << (l & 31));
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        for (int w = 0; w < nw; ++w) {
            const uint32_t word = flags[w];
            if (!word) continue;
            // lane i takes the i-th flagged atom of this word (ascending order)
            int l = -1;
            if (lane < __popc(word)) {
                uint32_t x = word;
                for (int s = 0; s < lane; ++s) x &= x - 1u;
                l = (w << 5) + __ffs(x) - 1;
            }
            int key = -1;
            float q = 0.f;
            if (l >= 0) {
                const float4 a = __ldg(&L.atom[l]);
                const int j = charge_cell(rot_x(m + 3, a.x, a.y, a.z), G.pad, G.gw, G.ng);
                const int k = charge_cell(rot_x(m + 6, a.x, a.y, a.z), G.pad, G.gw, G.ng);
                key = j * G.ng + k;
                q = a.w;
            }
            const uint32_t grp = __match_any_sync(0xffffffffu, key);
            const bool leader = (l >= 0) && (lane == __ffs(grp) - 1);
            float acc = 0.f;
            if (leader) acc = cell(key / G.ng, key % G.ng);
            for (int b = 0; b < 32; ++b) {
                const float qb = __shfl_sync(0xffffffffu, q, b);
                if (leader && ((grp >> b) & 1u)) acc = __fadd_rn(acc, qb);
            }
            if (leader) cell(key / G.ng, key % G.ng) = acc;
            __syncwarp();
        }
    }
    __syncthreads();
}

// ------------------------------------------------------------------ K1
// MODE 0: ligand rotation + voxelization, store spectrum planes A.
// MODE 1: receptor grids (re, im) loaded from global, store spectrum planes A.
// MODE 2: ligand rotation + voxelization, store the voxel plane itself
//         (ng x ng real and imaginary parts) for parity checks; no FFT.
template <int N, int MODE>
__global__ void __launch_bounds__(kNT, 1)
    k_plane_fwd(LigandView L, GridView G, const float *__restrict__ rotm, const float *__restrict__ src_r,
                const float *__restrict__ src_i, float2 *__restrict__ A, float *__restrict__ vox_r,
                float *__restrict__ vox_i) {
    constexpr int NG = N / 2, OFF = N / 4, PITCH = N + 1;
    constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *S = reinterpret_cast<float2 *>(smem_raw);                      // N x PITCH
    uint32_t *flags = reinterpret_cast<uint32_t *>(S + (size_t)N * PITCH); // atom bitmap
    __shared__ VoxShared<NG> vs;
    __shared__ float m[9];

    const int p = blockIdx.x;
    const int b = blockIdx.y;
    const int tid = threadIdx.x;

    if (MODE == 1) {
        for (int c = tid; c < NG * NG; c += blockDim.x) {
            const int q = c / NG, s = c % NG;
            const size_t gidx = ((size_t)p * NG + q) * NG + s;
            S[(q + OFF) * PITCH + s + OFF] = make_float2(src_r[gidx], src_i[gidx]);
        }
        __syncthreads();
    } else {
        if (tid < 9) m[tid] = rotm[(size_t)b * 9 + tid];
        for (int w = tid; w < 5 * NG * VoxShared<NG>::W; w += blockDim.x) (&vs.core[0][0])[w] = 0u;
        for (int w = tid; w < 3 * NG * VoxShared<NG>::W; w += blockDim.x) (&vs.surf[0][0])[w] = 0u;
        __syncthreads();
        const bool gd = (L.delta != 1.0f);
        vox_mark<NG>(vs, L, G, m, p, gd);
        __syncthreads();
        for (int c = tid; c < NG * NG; c += blockDim.x) {
            const int q = c / NG, s = c % NG;
            S[(q + OFF) * PITCH + s + OFF] = make_float2(vox_real<NG>(vs, p, q, s, NG, L.delta, gd), 0.f);
        }
        __syncthreads();
        vox_charges(flags, L, G, m, p,
                    [&](int q, int s) -> float & { return S[(q + OFF) * PITCH + s + OFF].y; });
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
        fft_phase1<N, -1, true>(S + (q + OFF) * PITCH, 1, t, G.tw);
    }
    __syncthreads();
    {
        constexpr int IPT = (NG * R1 + kNT - 1) / kNT;
        float2 reg[IPT][R2];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = tid + r * kNT;
            if (it < NG * R1) fft_phase2<N, -1>(S + ((it % NG) + OFF) * PITCH, 1, it / NG, reg[r]);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = tid + r * kNT;
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
        fft_phase1<N, -1, true>(S + c, PITCH, t, G.tw);
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

// ------------------------------------------------------------------ K2
// MODE 0: forward x-FFT, conj(R^) product, inverse x-FFT -> G.
// MODE 1: forward x-FFT only -> R^ (receptor spectrum, written to `out`).
template <int N, int MODE>
__global__ void __launch_bounds__(kNT)
    k_xline(GridView G, const float2 *__restrict__ A, const float2 *__restrict__ Rh, float2 *__restrict__ out) {
    constexpr int NG = N / 2, OFF = N / 4;
    constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
    __shared__ float2 X[N * kLT];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarp = blockDim.x >> 5;
    constexpr int TILES = N / kLT;
    const int ky = blockIdx.x / TILES;
    const int kz0 = (blockIdx.x % TILES) * kLT;
    const int b = blockIdx.y;

    const float2 *Ab = A + (size_t)b * NG * N * N;
    for (int pp = warp; pp < NG; pp += nwarp)
        X[(pp + OFF) * kLT + lane] = Ab[((size_t)pp * N + ky) * N + kz0 + lane];
    __syncthreads();
    for (int it = threadIdx.x; it < kLT * R2; it += blockDim.x)
        fft_phase1<N, -1, true>(X + (it % kLT), kLT, it / kLT, G.tw);
    __syncthreads();

    constexpr int IPT = (kLT * R1 + kNT - 1) / kNT;
    if (MODE == 1) {
        for (int it = threadIdx.x; it < kLT * R1; it += blockDim.x) {
            const int ln = it % kLT, u = it / kLT;
            float2 o[R2];
            fft_phase2<N, -1>(X + ln, kLT, u, o);
            static_for<0, R2>([&](auto k2) {
                const int kx = u + R1 * k2;
                out[((size_t)kx * N + ky) * N + kz0 + ln] = o[k2];
            });
        }
        return;
    }
    {
        float2 reg[IPT][R2];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = threadIdx.x + r * blockDim.x;
            if (it < kLT * R1) {
                const int ln = it % kLT, u = it / kLT;
                fft_phase2<N, -1>(X + ln, kLT, u, reg[r]);
                static_for<0, R2>([&](auto k2) {
                    const int kx = u + R1 * k2;
                    const float2 rh = __ldg(&Rh[((size_t)kx * N + ky) * N + kz0 + ln]);
                    reg[r][k2] = cmulconj(rh, reg[r][k2]);
                });
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = threadIdx.x + r * blockDim.x;
            if (it < kLT * R1) {
                const int ln = it % kLT, u = it / kLT;
                static_for<0, R2>([&](auto k2) { X[(u + R1 * k2) * kLT + ln] = reg[r][k2]; });
            }
        }
    }
    __syncthreads();
    for (int it = threadIdx.x; it < kLT * R2; it += blockDim.x)
        fft_phase1<N, +1, false>(X + (it % kLT), kLT, it / kLT, G.tw);
    __syncthreads();
    float2 *Gb = out + (size_t)b * N * N * N;
    for (int it = threadIdx.x; it < kLT * R1; it += blockDim.x) {
        const int ln = it % kLT, u = it / kLT;
        float2 o[R2];
        fft_phase2<N, +1>(X + ln, kLT, u, o);
        static_for<0, R2>([&](auto k2) {
            const int x = u + R1 * k2;
            Gb[((size_t)x * N + ky) * N + kz0 + ln] = o[k2];
        });
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

// Block-wide best candidate strictly after (pk, pi) in selection order.
__device__ __forceinline__ Cand block_best(Cand mine, Cand *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float k2 = __shfl_down_sync(0xffffffffu, mine.key, o);
        const int i2 = __shfl_down_sync(0xffffffffu, mine.idx, o);
        if (i2 >= 0 && (mine.idx < 0 || key_better(k2, i2, mine.key, mine.idx))) {
            mine.key = k2;
            mine.idx = i2;
        }
    }
    if (lane == 0) red[warp] = mine;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        Cand c = (lane < nw) ? red[lane] : Cand{0.f, -1};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float k2 = __shfl_down_sync(0xffffffffu, c.key, o);
            const int i2 = __shfl_down_sync(0xffffffffu, c.idx, o);
            if (i2 >= 0 && (c.idx < 0 || key_better(k2, i2, c.key, c.idx))) {
                c.key = k2;
                c.idx = i2;
            }
        }
        if (lane == 0) red[32] = c;
    }
    __syncthreads();
    const Cand r = red[32];
    __syncthreads();
    return r;
}

// Candidates are written as (key, linear index); key = raw real part when
// t == 1 and raw / nf3 otherwise (src/fft_process.cpp:415, :437).
template <int N>
__global__ void __launch_bounds__(kNT, 1)
    k_plane_inv(GridView G, const float2 *__restrict__ Gsp, int t, float nf3f, Cand *__restrict__ cand) {
    constexpr int PITCH = N + 1;
    constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *S = reinterpret_cast<float2 *>(smem_raw);
    float *SC = reinterpret_cast<float *>(smem_raw);
    __shared__ Cand red[33];
    const int x = blockIdx.x;
    const int b = blockIdx.y;
    const int tid = threadIdx.x;

    const float2 *Gp = Gsp + ((size_t)b * N + x) * N * N;
    for (int e = tid; e < N * N; e += blockDim.x) S[(e / N) * PITCH + (e % N)] = Gp[e];
    __syncthreads();
    // inverse y: columns (lanes = kz)
    for (int it = tid; it < N * R2; it += blockDim.x)
        fft_phase1<N, +1, false>(S + (it % N), PITCH, it / N, G.tw);
    __syncthreads();
    constexpr int IPT = (N * R1 + kNT - 1) / kNT;
    {
        float2 reg[IPT][R2];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = tid + r * kNT;
            if (it < N * R1) fft_phase2<N, +1>(S + (it % N), PITCH, it / N, reg[r]);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = tid + r * kNT;
            if (it < N * R1) {
                const int c = it % N, u = it / N;
                static_for<0, R2>([&](auto k2) { S[(u + R1 * k2) * PITCH + c] = reg[r][k2]; });
            }
        }
    }
    __syncthreads();
    // inverse z: rows (lanes = y)
    for (int it = tid; it < N * R2; it += blockDim.x)
        fft_phase1<N, +1, false>(S + (it % N) * PITCH, 1, it / N, G.tw);
    __syncthreads();
    {
        float reg[IPT][R2];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = tid + r * kNT;
            if (it < N * R1) {
                float2 o[R2];
                fft_phase2<N, +1>(S + (it % N) * PITCH, 1, it / N, o);
                static_for<0, R2>([&](auto k2) {
                    reg[r][k2] = (t == 1) ? o[k2].x : __fdiv_rn(o[k2].x, nf3f);
                });
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const int it = tid + r * kNT;
            if (it < N * R1) {
                const int y = it % N, u = it / N;
                static_for<0, R2>([&](auto k2) { SC[y * N + u + R1 * k2] = reg[r][k2]; });
            }
        }
    }
    __syncthreads();
    // t rounds of block-wide selection
    Cand prev{0.f, -1};
    Cand *out = cand + ((size_t)b * N + x) * t;
    for (int round = 0; round < t; ++round) {
        Cand mine{0.f, -1};
        for (int e = tid; e < N * N; e += blockDim.x) {
            const float k = SC[e];
            if (!(k == k)) continue;   // NaN
            const int idx = x * N * N + e;
            if (prev.idx >= 0 && !key_better(prev.key, prev.idx, k, idx)) continue;
            if (mine.idx < 0 || key_better(k, idx, mine.key, mine.idx)) {
                mine.key = k;
                mine.idx = idx;
            }
        }
        prev = block_best(mine, red);
        if (tid == 0) out[round] = prev;
        if (prev.idx < 0) {
            // nothing left: fill the remaining slots as empty
            if (tid == 0)
                for (int r2 = round + 1; r2 < t; ++r2) out[r2] = Cand{0.f, -1};
            break;
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
                if (idx < 0 || !(prev.key > -99999.0f)) {
                    score = -99999.0f;
                    idx = 0;
                } else {
                    score = prev.key;
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
