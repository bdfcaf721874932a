// Receptor grids on the GPU (sm_100a), bit-exact with MEGADOCK's CPU code
// (Receptor::rpscace, src/receptor.cpp:20-254; Receptor::electro, :258-346).
//
//   K_r0 k_rec_prep    per atom: centre cell, squared radii, ACE term, field reach
//   K_r1 k_rec_core    per atom: core value in the cube of +-reach cells within 1.5 R^2
//   K_r2 k_rec_rays    per line and axis: open space reachable straight from a face
//   K_r3 k_rec_sweep   two in-place 6-neighbour propagation sweeps (see below)
//   K_r4 k_rec_final   cavities -> core, open space -> 0
//   K_r5 k_rec_rows    per (i, j) row, the atoms whose shell reaches it, in atom order
//   K_r6 k_rec_shell   per cell: sum over those atoms of 1 - 0.8 ACE (double, rounded per add)
//   K_r7 k_rec_planes  per x plane, the charged atoms whose cube reaches it, in atom order
//   K_r8 k_rec_elec    per non-core cell: sum over those atoms of e beta q / eps(r) / r
//
// Every float operation is an explicitly rounded intrinsic in the reference's
// association order, and every sum runs over atoms in ascending order, so the
// grids equal the sequential CPU result.
//
// The propagation sweep visits cells in linear order c = (i, j, k) and, for an
// open cell with 1 <= i <= ng-2 and 2 <= j, k <= ng-2 ("valid"), opens its zero
// neighbours.  A cell is open when the sweep reaches it iff it was open at the
// start, or it was zero and one of its predecessors (k-1, j-1 or i-1 on the
// same lines) is valid and open when visited:
//     R(c) = O(c) | (Z(c) & OR_p (V(p) & R(p)))
// which depends only on rows (i, j-1) and (i-1, j) and on the row itself, so
// rows on the same anti-diagonal i + j are independent: one CTA walks the
// 2 ng - 1 anti-diagonals, a warp per row, R kept as bit masks in shared
// memory.  Zero cells next to a valid open successor (k+1, j+1 or i+1) are
// opened too, after their own visit, so they do not propagate in that sweep.
#pragma once
#include <cstdint>

namespace mdb {

// Row masks of the propagation sweep: ceil(ng / 64) 64-bit words per (i, j)
// row.  Up to ng = 112 every row's mask fits one CTA's shared memory (two
// words, 16 B x 112^2); larger grids keep them in a global scratch buffer.
constexpr int kRecSmemNg = 112;
constexpr int kRecMaxNg = 256;

struct RecAtom {
    float x, y, z;
    int io, jo, ko;       // centre cell, (int)(c / gw + ng/2)
    int iw, jw, kw;       // centre cell of the field, (int)(c / width + ng/2)
    float core2, shell2;  // 1.5 R^2 and (R + 3.6)^2
    double term;          // 1 + ACE (-0.8) ratio
    float q;
    int reach_e;          // field cube half width (-1: uncharged)
};

struct RecParams {
    int ng, na;
    float gw, width, eps_core, e_ratio, cpg;   // cpg: charge per grid cell
    double ace_ratio;
    int reach_core, reach_shell;
};

__device__ __forceinline__ float rec_sq(float c, float g) {
    const float d = __fsub_rn(c, g);
    return __fmul_rn(d, d);
}

__global__ void k_rec_prep(RecParams P, const float *__restrict__ xyz, const float *__restrict__ radius,
                           const float *__restrict__ charge, const float *__restrict__ ace, RecAtom *__restrict__ A) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= P.na) return;
    RecAtom a;
    a.x = xyz[3 * l];
    a.y = xyz[3 * l + 1];
    a.z = xyz[3 * l + 2];
    const float half = (float)(P.ng / 2);
    a.io = __float2int_rz(__fadd_rn(__fdiv_rn(a.x, P.gw), half));
    a.jo = __float2int_rz(__fadd_rn(__fdiv_rn(a.y, P.gw), half));
    a.ko = __float2int_rz(__fadd_rn(__fdiv_rn(a.z, P.gw), half));
    a.iw = __float2int_rz(__fadd_rn(__fdiv_rn(a.x, P.width), half));
    a.jw = __float2int_rz(__fadd_rn(__fdiv_rn(a.y, P.width), half));
    a.kw = __float2int_rz(__fadd_rn(__fdiv_rn(a.z, P.width), half));
    const float r = radius[l];
    a.core2 = __fmul_rn(__fmul_rn(r, r), 1.5f);
    const float rd = __fadd_rn(r, 3.6f);
    a.shell2 = __fmul_rn(rd, rd);
    a.term = __dadd_rn(1.0, __dmul_rn(__dmul_rn((double)ace[l], -0.8), P.ace_ratio));
    const float q = charge[l];
    const float aq = fabsf(q);
    a.q = q;
    if (aq <= 1.0e-6f) a.reach_e = -1;
    else if ((double)aq < 0.07) a.reach_e = 4;
    else if ((double)aq < 0.21) a.reach_e = 5;
    else a.reach_e = __float2int_rz(__fdiv_rn(aq, P.cpg));
    A[l] = a;
}

__global__ void k_rec_core(RecParams P, const RecAtom *__restrict__ A, const float *__restrict__ gc,
                           float *__restrict__ grid) {
    const int l = blockIdx.x;
    const RecAtom a = A[l];
    const int ng = P.ng, R = P.reach_core;
    const int i0 = max(a.io - R, 0), i1 = min(a.io + R + 1, ng);
    const int j0 = max(a.jo - R, 0), j1 = min(a.jo + R + 1, ng);
    const int k0 = max(a.ko - R, 0), k1 = min(a.ko + R + 1, ng);
    const int ni = max(i1 - i0, 0), nj = max(j1 - j0, 0), nk = max(k1 - k0, 0);
    for (int t = threadIdx.x; t < ni * nj * nk; t += blockDim.x) {
        const int i = i0 + t / (nj * nk), j = j0 + (t / nk) % nj, k = k0 + t % nk;
        const float d = __fadd_rn(__fadd_rn(rec_sq(a.x, gc[i]), rec_sq(a.y, gc[j])), rec_sq(a.z, gc[k]));
        if (d < a.core2) grid[((size_t)i * ng + j) * ng + k] = P.eps_core;
    }
}

// one thread per (a, b, axis): walk in from both faces until a core cell
__global__ void k_rec_rays(RecParams P, float *__restrict__ grid, float open_space) {
    const int ng = P.ng;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * ng * ng) return;
    const int ax = t / (ng * ng), a = (t / ng) % ng, b = t % ng;
    const size_t ng2 = (size_t)ng * ng;
    size_t base, step;
    if (ax == 0) {
        base = (size_t)a + (size_t)ng * b;
        step = ng2;
    } else if (ax == 1) {
        base = (size_t)b * ng2 + (size_t)a * ng;
        step = 1;
    } else {
        base = (size_t)a * ng2 + b;
        step = ng;
    }
    for (int k = 0; k < ng; ++k) {
        float *v = &grid[base + step * k];
        if (*v == P.eps_core) break;
        *v = open_space;
    }
    for (int k = ng - 1; k >= 0; --k) {
        float *v = &grid[base + step * k];
        if (*v == P.eps_core) break;
        *v = open_space;
    }
}

template <int WORDS>
struct RowMask {
    unsigned long long w[WORDS];
};

template <int WORDS>
__device__ __forceinline__ bool mbit(const RowMask<WORDS> &m, int k) {
    return (m.w[k >> 6] >> (k & 63)) & 1ull;
}

// One propagation sweep; one CTA.  The R masks of every row (ng^2 of them)
// live in dynamic shared memory, or with GMEM in `gmask` (ng^2 entries).
template <int WORDS, bool GMEM>
__global__ void __launch_bounds__(1024)
    k_rec_sweep(RecParams P, float *__restrict__ grid, float open_space, RowMask<WORDS> *__restrict__ gmask) {
    extern __shared__ __align__(16) unsigned char rec_smem[];
    RowMask<WORDS> *Rm = GMEM ? gmask : reinterpret_cast<RowMask<WORDS> *>(rec_smem);
    const int ng = P.ng;
    const size_t ng2 = (size_t)ng * ng;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    auto vrow = [&](int i, int j) { return i >= 1 && i <= ng - 2 && j >= 2 && j <= ng - 2; };
    for (int d = 0; d <= 2 * (ng - 1); ++d) {
        const int ilo = max(0, d - (ng - 1)), ihi = min(ng - 1, d);
        for (int i = ilo + warp; i <= ihi; i += nwarps) {
            const int j = d - i;
            const float *row = grid + (size_t)i * ng2 + (size_t)j * ng;
            RowMask<WORDS> O{}, Z{};
            for (int k0 = 0; k0 < ng; k0 += 32) {
                const int k = k0 + lane;
                const float v = k < ng ? row[k] : 1.0f;
                const unsigned o = __ballot_sync(0xffffffffu, k < ng && v == open_space);
                const unsigned z = __ballot_sync(0xffffffffu, k < ng && v == 0.0f);
                O.w[k0 >> 6] |= (unsigned long long)o << (k0 & 63);
                Z.w[k0 >> 6] |= (unsigned long long)z << (k0 & 63);
            }
            if (lane == 0) {
                RowMask<WORDS> In{};
                if (j > 0 && vrow(i, j - 1)) {
                    const RowMask<WORDS> q = Rm[(size_t)i * ng + j - 1];
#pragma unroll
                    for (int w = 0; w < WORDS; ++w) In.w[w] |= q.w[w];
                }
                if (i > 0 && vrow(i - 1, j)) {
                    const RowMask<WORDS> q = Rm[(size_t)(i - 1) * ng + j];
#pragma unroll
                    for (int w = 0; w < WORDS; ++w) In.w[w] |= q.w[w];
                }
                const bool vr = vrow(i, j);
                // Vk: positions 2 <= k <= ng - 2 (as a source on the k axis)
                RowMask<WORDS> Vk{};
#pragma unroll
                for (int w = 0; w < WORDS; ++w) {
                    const int lo = max(2 - 64 * w, 0), hi = min(ng - 2 - 64 * w, 63);   // bit range in word w
                    if (hi >= lo)
                        Vk.w[w] = ((hi - lo == 63) ? ~0ull : ((1ull << (hi - lo + 1)) - 1ull)) << lo;
                }
                // seeds S = O | (Z & In & Vk); k receives from k - 1 when
                // P(k) = Z(k) & Vk(k - 1) & vr.  R = S | (P & (R << 1)) is a
                // carry chain: within a run of P, everything from the first
                // position after a reached cell up to the run's end is reached,
                // i.e. P & (~(P + B) | B) with B = (R << 1) & P restricted to
                // the seeds (the addition carries through the run); a run
                // crossing a word boundary takes the previous word's top bit
                // of R as its carry in.
                RowMask<WORDS> R{};
                unsigned long long carry = 0ull;   // R at bit 63 of the previous word
#pragma unroll
                for (int w = 0; w < WORDS; ++w) {
                    const unsigned long long S = O.w[w] | (Z.w[w] & In.w[w] & Vk.w[w]);
                    const unsigned long long vprev = (Vk.w[w] << 1) | (w ? (Vk.w[w - 1] >> 63) : 0ull);
                    const unsigned long long P = vr ? (Z.w[w] & vprev) : 0ull;
                    const unsigned long long B = ((S << 1) | carry) & P;
                    const unsigned long long r = S | (P & (~(P + B) | B));
                    R.w[w] = r;
                    carry = r >> 63;
                }
                Rm[(size_t)i * ng + j] = R;
            }
            __syncwarp();
        }
        __syncthreads();
    }
    // apply: forward-reached cells, then zero cells with a valid reached successor
    for (size_t c = threadIdx.x; c < ng2 * ng; c += blockDim.x) {
        const int i = (int)(c / ng2), j = (int)((c / ng) % ng), k = (int)(c % ng);
        const RowMask<WORDS> &r = Rm[(size_t)i * ng + j];
        if (mbit(r, k)) continue;   // written below, after every read of this sweep
        if (grid[c] != 0.0f) continue;
        bool b = false;
        if (k + 1 < ng && vrow(i, j) && k + 1 >= 2 && k + 1 <= ng - 2 && mbit(r, k + 1)) b = true;
        if (!b && j + 1 < ng && vrow(i, j + 1) && k >= 2 && k <= ng - 2 && mbit(Rm[(size_t)i * ng + j + 1], k)) b = true;
        if (!b && i + 1 < ng && vrow(i + 1, j) && k >= 2 && k <= ng - 2 && mbit(Rm[(size_t)(i + 1) * ng + j], k)) b = true;
        if (b) grid[c] = open_space;
    }
    __syncthreads();
    for (size_t c = threadIdx.x; c < ng2 * ng; c += blockDim.x) {
        const int i = (int)(c / ng2), j = (int)((c / ng) % ng), k = (int)(c % ng);
        if (mbit(Rm[(size_t)i * ng + j], k)) grid[c] = open_space;
    }
}

__global__ void k_rec_final(RecParams P, float *__restrict__ grid, float open_space) {
    const size_t ng3 = (size_t)P.ng * P.ng * P.ng;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < ng3; c += (size_t)gridDim.x * blockDim.x) {
        const float v = grid[c];
        if (v == 0.0f) grid[c] = P.eps_core;
        else if (v == open_space) grid[c] = 0.0f;
    }
}

// Atoms (in order) whose shell cube and sphere reach row (i, j): one warp per
// row, 32 atoms per step, compacted in order with a ballot.  count pass
// (out == nullptr) writes cnt[row]; fill pass writes out[start[row] ..].
__global__ void k_rec_rows(RecParams P, const RecAtom *__restrict__ A, const float *__restrict__ gc,
                           int *__restrict__ cnt, const int *__restrict__ start, int *__restrict__ out) {
    const int row = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int ng = P.ng;
    if (row >= ng * ng) return;   // whole warps
    const int i = row / ng, j = row % ng;
    const int R = P.reach_shell;
    int n = 0;
    const int base = out ? start[row] : 0;
    for (int l0 = 0; l0 < P.na; l0 += 32) {
        const int l = l0 + lane;
        bool hit = false;
        if (l < P.na) {
            const RecAtom &a = A[l];
            hit = !(i < a.io - R || i > a.io + R || j < a.jo - R || j > a.jo + R) &&
                  !(__fadd_rn(rec_sq(a.x, gc[i]), rec_sq(a.y, gc[j])) > a.shell2);
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (hit && out) out[base + n + __popc(m & ((1u << lane) - 1u))] = l;
        n += __popc(m);
    }
    if (!out && lane == 0) cnt[row] = n;
}

__global__ void k_rec_shell(RecParams P, const RecAtom *__restrict__ A, const float *__restrict__ gc,
                            const int *__restrict__ start, const int *__restrict__ list, float *__restrict__ grid) {
    const int ng = P.ng;
    const size_t ng3 = (size_t)ng * ng * ng;
    const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= ng3) return;
    const int i = (int)(c / ((size_t)ng * ng)), j = (int)((c / ng) % ng), k = (int)(c % ng);
    const int row = i * ng + j, R = P.reach_shell;
    float v = 0.f;
    for (int e = start[row]; e < start[row + 1]; ++e) {
        const RecAtom &a = A[list[e]];
        if (k < a.ko - R || k > a.ko + R) continue;
        const float d = __fadd_rn(__fadd_rn(rec_sq(a.x, gc[i]), rec_sq(a.y, gc[j])), rec_sq(a.z, gc[k]));
        if (d < a.shell2) v = __double2float_rn(__dadd_rn((double)v, a.term));
    }
    if (grid[c] != P.eps_core) grid[c] = v;
}

// Charged atoms (in order) whose field cube reaches plane i: one warp per plane.
__global__ void k_rec_planes(RecParams P, const RecAtom *__restrict__ A, int *__restrict__ cnt,
                             const int *__restrict__ start, int *__restrict__ out) {
    const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= P.ng) return;   // whole warps
    int n = 0;
    const int base = out ? start[i] : 0;
    for (int l0 = 0; l0 < P.na; l0 += 32) {
        const int l = l0 + lane;
        bool hit = false;
        if (l < P.na) {
            const RecAtom &a = A[l];
            hit = a.reach_e >= 0 && i >= a.iw - a.reach_e && i <= a.iw + a.reach_e;
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (hit && out) out[base + n + __popc(m & ((1u << lane) - 1u))] = l;
        n += __popc(m);
    }
    if (!out && lane == 0) cnt[i] = n;
}

__global__ void k_rec_elec(RecParams P, const RecAtom *__restrict__ A, const float *__restrict__ gc,
                           const int *__restrict__ start, const int *__restrict__ list,
                           const float *__restrict__ grid_r, float *__restrict__ grid_i) {
    const int ng = P.ng;
    const size_t ng3 = (size_t)ng * ng * ng;
    const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= ng3) return;
    float v = 0.f;
    if (!(grid_r[c] < 0.0f)) {   // receptor core cells carry no field
        const int i = (int)(c / ((size_t)ng * ng)), j = (int)((c / ng) % ng), k = (int)(c % ng);
        const float coef = __fmul_rn(P.e_ratio, -2800.0f);
        for (int e = start[i]; e < start[i + 1]; ++e) {
            const RecAtom &a = A[list[e]];
            if (j < a.jw - a.reach_e || j > a.jw + a.reach_e || k < a.kw - a.reach_e || k > a.kw + a.reach_e)
                continue;
            const float d2 = __fadd_rn(rec_sq(a.x, gc[i]), rec_sq(a.y, gc[j]));
            const float r = __fsqrt_rn(__fadd_rn(d2, rec_sq(a.z, gc[k])));
            float eps;
            if (r >= 8.0f) eps = 80.0f;
            else if (r > 6.0f) eps = __fadd_rn(__fmul_rn(38.0f, r), -224.0f);
            else eps = 4.0f;
            v = __fadd_rn(v, __fdiv_rn(__fdiv_rn(__fmul_rn(coef, a.q), eps), r));
        }
    }
    grid_i[c] = v;
}

}  // namespace mdb
