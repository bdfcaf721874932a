// Docking kernels for FFT edges above 224 (sm_100a), where one x-plane of
// the grid no longer fits one CTA's shared memory.  The same transforms as
// the plane kernels of dock_kernels.cuh, with the two axes of each plane
// transform done by separate launches through global memory:
//
//   K1r k_rows_fwd   (x-plane p, block of RB voxel rows): build the rows of
//                    the voxel plane (ligand classes + ordered charge sums,
//                    the receptor grids, or -- MODE 2 -- just store them) and
//                    run the pruned forward z-FFT of each row into A[p][y][kz]
//                    for the NG data rows y;
//   K1c k_cols_fwd   (x-plane p, block of CB columns kz): pruned forward y-FFT
//                    of the columns, in place in A -> A[p][ky][kz];
//   K2  k_xline_herm (unchanged): x-FFT, conj(R^) product, Hermitian fold,
//                    inverse x-FFT -> Gh[x][ky < N/2][kz];
//   K3r k_rows_inv   (x, block of RB rows ky): inverse z-FFT in place in Gh;
//   K3c k_cols_c2r   (x, block of CB columns z): unpack the half spectrum,
//                    N/2-point inverse along ky (real output), per-thread
//                    top-t lists, block merge -> candidates per (x, z block);
//   K4  k_merge      (unchanged) over N x ZB candidate groups per rotation.
//
// Each launch owns whole rows (K1r, K3r) or whole columns (K1c, K3c) of a
// plane: it reads every input of its rows or columns before a barrier and
// writes the results after it, so the in-place passes never race.
//
// References (MEGADOCK, akiyamalab): as the plane kernels -- embedding
// src/fft_process.cpp:306-330, FFT/product :333-396, top-t :399-458.
#pragma once
#include "dock_kernels.cuh"

namespace mdb {

constexpr int kNTS = 256;   // threads per CTA of the staged kernels
constexpr int kRB = 16;     // voxel rows / spectrum rows per CTA of K1r and K3r
constexpr int kCB = 16;     // columns per CTA of K1c and K3c

// largest edge whose plane kernels keep a whole plane in shared memory
constexpr int kMaxResidentN = 224;

template <int N>
constexpr bool staged() {
    return N > kMaxResidentN;
}

// column blocks of K3c per x-plane: candidate groups per plane
template <int N>
constexpr int c2r_zblocks() {
    return (N + kCB - 1) / kCB;
}

constexpr size_t rows_smem(int N) { return (size_t)kRB * (N + 1) * sizeof(float2); }
constexpr size_t cols_fwd_smem(int N) { return (size_t)N * (kCB + 1) * sizeof(float2); }
constexpr size_t cols_c2r_smem(int N) { return (size_t)(N / 2) * (kCB + 1) * sizeof(float2); }

// K1r.  Grid (NG planes, ceil(NG / RB) row blocks, nb), kNTS threads.
// MODE 0: ligand classes (K0 bit planes) and charged cells; MODE 1: receptor
// grids src_r / src_i ([NG][NG][NG] floats); MODE 2: store the voxel rows to
// vox_r / vox_i, no FFT.
template <int N, int MODE>
__global__ void __launch_bounds__(kNTS)
    k_rows_fwd(LigandView L, GridView G, const uint32_t *__restrict__ vbits, const int2 *__restrict__ qlist,
               const int *__restrict__ qcount, const float *__restrict__ src_r, const float *__restrict__ src_i,
               float2 *__restrict__ A, float *__restrict__ vox_r, float *__restrict__ vox_i) {
    constexpr int NG = N / 2, OFF = N / 4, PZ = N + 1;
    constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
    constexpr int W = VoxShared<NG>::W;
    constexpr bool PR = prune_ok<N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *Z = reinterpret_cast<float2 *>(smem_raw);   // RB rows x PZ
    const int p = blockIdx.x, q0 = blockIdx.y * kRB, b = blockIdx.z, tid = threadIdx.x;
    const int nr = min(kRB, NG - q0);
    if constexpr (!PR && MODE != 2) {
        // the unpruned z pass reads the padding columns: make them zero
        for (int c = tid; c < kRB * PZ; c += blockDim.x) Z[c] = make_float2(0.f, 0.f);
        __syncthreads();
    }
    if constexpr (MODE == 1) {
        for (int c = tid; c < nr * NG; c += blockDim.x) {
            const int r = c / NG, s = c % NG;
            const size_t gidx = ((size_t)p * NG + q0 + r) * NG + s;
            Z[r * PZ + s + OFF] = make_float2(src_r[gidx], src_i[gidx]);
        }
        __syncthreads();
    } else {
        const uint32_t *vb = vbits + ((size_t)b * NG + p) * 2 * NG * W;
        for (int c = tid; c < nr * NG; c += blockDim.x) {
            const int r = c / NG, s = c % NG, q = q0 + r;
            const uint32_t bit = 1u << (s & 31);
            const float v = (__ldg(&vb[q * W + (s >> 5)]) & bit) ? L.delta
                            : (__ldg(&vb[NG * W + q * W + (s >> 5)]) & bit) ? 1.0f : 0.0f;
            Z[r * PZ + s + OFF] = make_float2(v, 0.f);
        }
        __syncthreads();
        // charged cells of this plane whose row falls in the block
        const int nq = qcount[(size_t)b * NG + p];
        const int2 *ql = qlist + ((size_t)b * NG + p) * NG * NG;
        for (int e = tid; e < nq; e += blockDim.x) {
            const int2 c = ql[e];
            const int r = c.x / NG - q0;
            if ((unsigned)r < (unsigned)nr) Z[r * PZ + c.x % NG + OFF].y = __int_as_float(c.y);
        }
        __syncthreads();
        if constexpr (MODE == 2) {
            for (int c = tid; c < nr * NG; c += blockDim.x) {
                const int r = c / NG, s = c % NG;
                const float2 v = Z[r * PZ + s + OFF];
                const size_t gidx = (((size_t)b * NG + p) * NG + q0 + r) * NG + s;
                vox_r[gidx] = v.x;
                vox_i[gidx] = v.y;
            }
            return;
        }
    }
    // z-FFT of the block's rows: phase 1 in place, phase 2 to global (row y = q + OFF)
    for (int it = tid; it < nr * R2; it += blockDim.x) {
        const int t = it % R2, r = it / R2;
        fft_phase1<N, -1, PR>(Z + r * PZ, 1, t, G.tw);
    }
    __syncthreads();
    float2 *Ap = A + ((size_t)b * NG + p) * N * N;
    for (int it = tid; it < nr * R1; it += blockDim.x) {
        const int r = it / R1, u = it % R1;
        float2 o[R2];
        fft_phase2<N, -1>(Z + r * PZ, 1, u, o);
        float2 *dst = Ap + (size_t)(q0 + r + OFF) * N;
        static_for<0, R2>([&](auto k2) { dst[u + R1 * k2] = o[k2]; });
    }
}

// K1c.  Grid (NG planes, ceil(N / CB) column blocks, nb), kNTS threads.
// Rows y outside [OFF, OFF + NG) of the z-transformed plane are zero (K1r
// writes only the data rows); the pruned pass never reads them and the
// unpruned one substitutes zeros.
template <int N>
__global__ void __launch_bounds__(kNTS) k_cols_fwd(GridView G, float2 *__restrict__ A) {
    constexpr int NG = N / 2, OFF = N / 4, PB = kCB + 1;
    constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
    constexpr bool PR = prune_ok<N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *Y = reinterpret_cast<float2 *>(smem_raw);   // N rows x PB
    const int p = blockIdx.x, c0 = blockIdx.y * kCB, b = blockIdx.z, tid = threadIdx.x;
    const int nc = min(kCB, N - c0);
    float2 *Ap = A + ((size_t)b * NG + p) * N * N + c0;
    for (int it = tid; it < nc * R2; it += blockDim.x) {
        const int t = it / nc, c = it % nc;
        float2 v[R1];
        static_for<0, R1>([&](auto m_) {
            constexpr int m = decltype(m_)::value;
            const int y = t + R2 * m;
            if constexpr (PR && (m < R1 / 4 || m >= 3 * R1 / 4)) {
                v[m] = make_float2(0.f, 0.f);
            } else if constexpr (PR) {
                v[m] = Ap[(size_t)y * N + c];
            } else {
                v[m] = ((unsigned)(y - OFF) < (unsigned)NG) ? Ap[(size_t)y * N + c] : make_float2(0.f, 0.f);
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
    for (int it = tid; it < nc * R1; it += blockDim.x) {
        const int u = it / nc, c = it % nc;
        float2 o[R2];
        fft_phase2<N, -1>(Y + c, PB, u, o);
        static_for<0, R2>([&](auto k2) { Ap[(size_t)(u + R1 * k2) * N + c] = o[k2]; });
    }
}

// K3r.  Grid (N planes x, ceil(N/2 / RB) row blocks, nb), kNTS threads:
// inverse z-FFT of rows ky of Gh[x][ky < N/2][kz], in place.
template <int N>
__global__ void __launch_bounds__(kNTS) k_rows_inv(GridView G, float2 *__restrict__ Gh) {
    constexpr int NH = N / 2, PZ = N + 1;
    constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *Z = reinterpret_cast<float2 *>(smem_raw);   // RB rows x PZ
    const int x = blockIdx.x, q0 = blockIdx.y * kRB, b = blockIdx.z, tid = threadIdx.x;
    const int nr = min(kRB, NH - q0);
    float2 *Gp = Gh + ((size_t)b * N + x) * NH * N + (size_t)q0 * N;
    for (int it = tid; it < nr * R2; it += blockDim.x) {
        const int t = it % R2, r = it / R2;   // lanes along z: coalesced row loads
        float2 v[R1];
        static_for<0, R1>([&](auto m_) {
            constexpr int mm = decltype(m_)::value;
            v[mm] = Gp[(size_t)r * N + t + R2 * mm];
        });
        Dft<R1, +1>::run(v);
        static_for<0, R1>([&](auto k1_) {
            constexpr int k1 = decltype(k1_)::value;
            float2 xv = v[k1];
            if constexpr (k1 != 0) xv = cmul(xv, conjf2(__ldg(&G.tw[t * k1])));
            Z[r * PZ + k1 * R2 + t] = xv;
        });
    }
    __syncthreads();
    for (int it = tid; it < nr * R1; it += blockDim.x) {
        const int r = it / R1, u = it % R1;
        float2 o[R2];
        fft_phase2<N, +1>(Z + r * PZ, 1, u, o);
        static_for<0, R2>([&](auto k2) { Gp[(size_t)r * N + u + R1 * k2] = o[k2]; });
    }
}

// K3c.  Grid (N planes x, ZB column blocks, nb), kNTS threads.  Input: Gh
// after K3r (row 0 holds h0 + i h_{N/2}, both real).  Per column z of the
// block: Z[k] = (X[k] + conj X[N/2-k]) + i w^k (X[k] - conj X[N/2-k]),
// w = e^{2 pi i/N}, whose N/2-point inverse FFT is s[2m] + i s[2m+1]; the
// scores feed per-thread top-T lists (after `floor` when a later pass of T),
// merged into this block's candidates
// cand[((b*N + x)*ZB + zb)*t + out0 + j], j < nsel.
template <int N, int T>
__global__ void __launch_bounds__(kNTS)
    k_cols_c2r(GridView G, const float2 *__restrict__ Gh, int t, int out0, int nsel, Cand *__restrict__ cand) {
    constexpr int NH = N / 2, PS = kCB + 1, ZB = c2r_zblocks<N>();
    constexpr int Q1 = Plan<NH>::R1, Q2 = Plan<NH>::R2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *S = reinterpret_cast<float2 *>(smem_raw);   // NH rows x PS
    __shared__ Cand red[33];
    const int x = blockIdx.x, zb = blockIdx.y, b = blockIdx.z, tid = threadIdx.x;
    const int z0 = zb * kCB, nc = min(kCB, N - z0);
    Cand *out = cand + (((size_t)b * N + x) * ZB + zb) * t + out0;
    Cand floor{0.f, -1};
    if (out0 > 0) {
        floor = out[-1];
        if (floor.idx < 0) {   // an earlier pass already ran out of cells
            if (tid == 0)
                for (int r = 0; r < nsel; ++r) out[r] = Cand{0.f, -1};
            return;
        }
    }
    const float2 *Gp = Gh + ((size_t)b * N + x) * NH * N + z0;
    for (int e = tid; e < NH * nc; e += blockDim.x) {
        const int k = e / nc, c = e % nc;
        S[k * PS + c] = Gp[(size_t)k * N + c];
    }
    __syncthreads();
    // fold the half spectrum into Z, in place (pairs k, N/2-k)
    for (int it = tid; it < nc * (NH / 2 + 1); it += blockDim.x) {
        const int c = it % nc, k = it / nc;
        if (k == 0) {
            const float2 v = S[c];
            S[c] = make_float2(v.x + v.y, v.x - v.y);
        } else {
            const int k2 = NH - k;
            const float2 a = S[k * PS + c], cc = S[k2 * PS + c];
            const float2 wk = conjf2(__ldg(&G.tw[k])), wk2 = conjf2(__ldg(&G.tw[k2]));
            const float2 e1 = make_float2(a.x + cc.x, a.y - cc.y), d1 = make_float2(a.x - cc.x, a.y + cc.y);
            const float2 o1 = cmul(wk, d1);
            const float2 z1 = make_float2(e1.x - o1.y, e1.y + o1.x);
            if (k2 != k) {
                const float2 e2 = make_float2(cc.x + a.x, cc.y - a.y), d2 = make_float2(cc.x - a.x, cc.y + a.y);
                const float2 o2 = cmul(wk2, d2);
                S[k2 * PS + c] = make_float2(e2.x - o2.y, e2.y + o2.x);
            }
            S[k * PS + c] = z1;
        }
    }
    __syncthreads();
    // N/2-point inverse along ky, pass 1 (lanes = columns), in place
    for (int it = tid; it < nc * Q2; it += blockDim.x) {
        const int c = it % nc, tt = it / nc;
        float2 v[Q1];
        static_for<0, Q1>([&](auto m_) {
            constexpr int mm = decltype(m_)::value;
            v[mm] = S[(tt + Q2 * mm) * PS + c];
        });
        Dft<Q1, +1>::run(v);
        static_for<0, Q1>([&](auto k1_) {
            constexpr int k1 = decltype(k1_)::value;
            float2 xv = v[k1];
            if constexpr (k1 != 0) xv = cmul(xv, conjf2(__ldg(&G.tw[2 * tt * k1])));
            S[(k1 * Q2 + tt) * PS + c] = xv;
        });
    }
    __syncthreads();
    // pass 2 -> scores s[2m], s[2m+1] -> per-thread top-T
    TopList<T> top;
    top.init();
    const int base = x * N * N + z0;
    auto scan = [&](auto floor_on) {
        constexpr bool FL = decltype(floor_on)::value;
        for (int it = tid; it < nc * Q1; it += blockDim.x) {
            const int c = it % nc, u = it / nc;
            float2 o[Q2];
            static_for<0, Q2>([&](auto n2_) {
                constexpr int n2 = decltype(n2_)::value;
                o[n2] = S[(u * Q2 + n2) * PS + c];
            });
            Dft<Q2, +1>::run(o);
            const int cell0 = base + 2 * u * N + c;
            static_for<0, Q2>([&](auto k2_) {
                constexpr int k2 = decltype(k2_)::value;
                constexpr int step = 2 * Q1 * k2 * N;
                top.template insert<FL>(o[k2].x, cell0 + step, floor);
                top.template insert<FL>(o[k2].y, cell0 + step + N, floor);
            });
        }
    };
    if (floor.idx >= 0) {
        scan(std::true_type{});
    } else {
        // First pass: as in k_plane_c2r, each thread keeps its maximum; the
        // largest over the warps of each warp's nsel-th largest lane maximum
        // bounds this block's nsel-th best key from below, and only the
        // threads at or above it recompute their items and enter those cells
        // in the lists (equal keys still compete on the index there).
        float tmax = -INFINITY;   // fmaxf drops NaN keys, which are never selected
        for (int it = tid; it < nc * Q1; it += blockDim.x) {
            const int c = it % nc, u = it / nc;
            float2 o[Q2];
            static_for<0, Q2>([&](auto n2_) {
                constexpr int n2 = decltype(n2_)::value;
                o[n2] = S[(u * Q2 + n2) * PS + c];
            });
            Dft<Q2, +1>::run(o);
            static_for<0, Q2>([&](auto k2_) {
                constexpr int k2 = decltype(k2_)::value;
                tmax = fmaxf(tmax, fmaxf(o[k2].x, o[k2].y));
            });
        }
        __shared__ float thr_w[kNTS / 32];
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
        if (tmax >= thr) {
            for (int it = tid; it < nc * Q1; it += blockDim.x) {
                const int c = it % nc, u = it / nc;
                const int cell0 = base + 2 * u * N + c;
                float2 o[Q2];
                static_for<0, Q2>([&](auto n2_) {
                    constexpr int n2 = decltype(n2_)::value;
                    o[n2] = S[(u * Q2 + n2) * PS + c];
                });
                Dft<Q2, +1>::run(o);
                static_for<0, Q2>([&](auto k2_) {
                    constexpr int k2 = decltype(k2_)::value;
                    constexpr int step = 2 * Q1 * k2 * N;
                    const float2 sc = o[k2];
                    if (sc.x >= thr) top.template insert<false>(sc.x, cell0 + step, floor);
                    if (sc.y >= thr) top.template insert<false>(sc.y, cell0 + step + N, floor);
                });
            }
        }
    }
    // block merge: nsel rounds of the block-wide best list head
    for (int r = 0; r < nsel; ++r) {
        const Cand c = block_best(top.head(), red);
        if (tid == 0) out[r] = c.idx >= 0 ? c : Cand{0.f, -1};
        if (c.idx < 0) {
            if (tid == 0)
                for (int r2 = r + 1; r2 < nsel; ++r2) out[r2] = Cand{0.f, -1};
            break;
        }
        if (top.i[0] == c.idx) top.pop();   // the owner (cell indices are unique)
    }
}

}  // namespace mdb
