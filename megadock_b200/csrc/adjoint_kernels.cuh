// Adjoint of a smooth loss over the per-rotation top-1 scores (sm_100a).
//
// With s_r = score_r(t*_r) = sum_x Rr(x) Lr_r(x + t*_r) + Ri(x) Li_r(x + t*_r)
// (circular FFT coordinates, src/fft_process.cpp:333-346 product + inverse
// FFT) and dL/ds_r = w_r, the gradients are transposed correlations that
// collapse to shifts at the selected translations:
//   dL/dR(x)    = sum_r w_r L_r(x + t*_r)        (k_adj_receptor: gather, rotations in order)
//   dL/dL_r(y)  = w_r R(y - t*_r)                (k_adj_ligand)
//   dL/dq_a     = sum_r w_r Ri(c_r(a) - t*_r)    (k_adj_charge: through the charge-cell assignment)
// Grids are the ng^3 voxel grids; their FFT embedding is at offset N/4 on each
// axis (src/fft_process.cpp:306-330).  Accumulation is FP32 in a fixed order.
#pragma once
#include "dock_kernels.cuh"

namespace mdb {

// Voxel index of the embedded grid at FFT position (a + d) mod N, or -1 when
// it falls in the zero padding.  a in [0, ng), d in [0, N), ng = N/2 and the
// embedding offset N/4, so a + N/4 + d < 2N and one conditional subtraction
// is the modulo.
__device__ __forceinline__ int adj_cell(int a, int d, int N, int ng) {
    int y = a + (N >> 2) + d;
    if (y >= N) y -= N;
    y -= N >> 2;
    return ((unsigned)y < (unsigned)ng) ? y : -1;
}

// (N - d) mod N for d in [0, N): the shift that undoes d.
__device__ __forceinline__ int adj_neg(int d, int N) { return d == 0 ? 0 : N - d; }

// dRr/dRi += sum over the chunk's rotations of w_r * (Lr_r, Li_r)(x + t*_r).
__global__ void k_adj_receptor(int N, int ng, int nb, const float *__restrict__ vr, const float *__restrict__ vi,
                               const int4 *__restrict__ shift, const float *__restrict__ w, float *__restrict__ dRr,
                               float *__restrict__ dRi) {
    const size_t ng3 = (size_t)ng * ng * ng;
    const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ng3) return;
    const int i = (int)(c / ((size_t)ng * ng)), j = (int)((c / ng) % ng), k = (int)(c % ng);
    float ar = dRr[c], ai = dRi[c];
    for (int r = 0; r < nb; ++r) {
        const float wr = __ldg(&w[r]);
        if (wr == 0.f) continue;
        const int4 t = __ldg(&shift[r]);
        const int yi = adj_cell(i, t.x, N, ng), yj = adj_cell(j, t.y, N, ng), yk = adj_cell(k, t.z, N, ng);
        if (yi < 0 || yj < 0 || yk < 0) continue;
        const size_t y = (size_t)r * ng3 + ((size_t)yi * ng + yj) * ng + yk;
        ar = fmaf(wr, __ldg(&vr[y]), ar);
        ai = fmaf(wr, __ldg(&vi[y]), ai);
    }
    dRr[c] = ar;
    dRi[c] = ai;
}

// dL/dL_r(y) = w_r * R(y - t*_r) for the selected rotations (sel[m] = r).
__global__ void k_adj_ligand(int N, int ng, int nsel, const int *__restrict__ sel, const float *__restrict__ recr,
                             const float *__restrict__ reci, const int4 *__restrict__ shift,
                             const float *__restrict__ w, float *__restrict__ dLr, float *__restrict__ dLi) {
    const size_t ng3 = (size_t)ng * ng * ng;
    const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (c >= ng3 || m >= nsel) return;
    const int r = sel[m];
    const int i = (int)(c / ((size_t)ng * ng)), j = (int)((c / ng) % ng), k = (int)(c % ng);
    const int4 t = shift[r];
    const int xi = adj_cell(i, adj_neg(t.x, N), N, ng), xj = adj_cell(j, adj_neg(t.y, N), N, ng),
              xk = adj_cell(k, adj_neg(t.z, N), N, ng);
    float gr = 0.f, gi = 0.f;
    if (xi >= 0 && xj >= 0 && xk >= 0 && w[r] != 0.f) {
        const size_t x = ((size_t)xi * ng + xj) * ng + xk;
        gr = w[r] * recr[x];
        gi = w[r] * reci[x];
    }
    dLr[(size_t)m * ng3 + c] = gr;
    dLi[(size_t)m * ng3 + c] = gi;
}

// dL/dq_a = sum_r w_r Ri(c_r(a) - t*_r), c_r(a) = the atom's charge cell in
// rotation r (the same bit-exact rotation and cell rule as the voxelizer).
// One warp per atom: lane l sums rotations l, l + 32, ... in order, then a
// fixed shuffle tree adds the lanes, so the result does not depend on
// scheduling.
__global__ void k_adj_charge(LigandView L, GridView G, int N, int n_rot, const float *__restrict__ rotm,
                             const int4 *__restrict__ shift, const float *__restrict__ w,
                             const float *__restrict__ reci, float *__restrict__ dq) {
    const int a = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (a >= L.na) return;   // whole warps leave together
    const float4 at = __ldg(&L.atom[a]);
    const int ng = G.ng;
    float acc = 0.f;
    for (int r = lane; r < n_rot; r += 32) {
        const float wr = __ldg(&w[r]);
        if (wr == 0.f) continue;
        const float *m = rotm + 9 * (size_t)r;
        float mm[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) mm[e] = __ldg(&m[e]);
        const int ci = charge_cell(rot_x(mm, at.x, at.y, at.z), G.pad, G.gw, ng);
        const int cj = charge_cell(rot_x(mm + 3, at.x, at.y, at.z), G.pad, G.gw, ng);
        const int ck = charge_cell(rot_x(mm + 6, at.x, at.y, at.z), G.pad, G.gw, ng);
        const int4 t = __ldg(&shift[r]);
        const int xi = adj_cell(ci, adj_neg(t.x, N), N, ng), xj = adj_cell(cj, adj_neg(t.y, N), N, ng),
                  xk = adj_cell(ck, adj_neg(t.z, N), N, ng);
        if (xi < 0 || xj < 0 || xk < 0) continue;
        acc = fmaf(wr, __ldg(&reci[((size_t)xi * ng + xj) * ng + xk]), acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) dq[a] = acc;
}

// Score of one pose per block: sum_x Rr(x) Lr(x + t) + Ri(x) Li(x + t) over the
// receptor grid (the value the inverse FFT gives at translation t, formed
// directly).  Per-thread float sums in a fixed stride order, then a fixed
// shuffle tree, so the result does not depend on scheduling.
__global__ void k_pose_dot(int N, int ng, const float *__restrict__ recr, const float *__restrict__ reci,
                           const float *__restrict__ vr, const float *__restrict__ vi,
                           const int4 *__restrict__ shift, float *__restrict__ score) {
    __shared__ float part[32];
    const size_t ng3 = (size_t)ng * ng * ng;
    const int b = blockIdx.x;
    const int4 t = shift[b];
    const float *lr = vr + (size_t)b * ng3, *li = vi + (size_t)b * ng3;
    float acc = 0.f;
    for (size_t c = threadIdx.x; c < ng3; c += blockDim.x) {
        const int i = (int)(c / ((size_t)ng * ng)), j = (int)((c / ng) % ng), k = (int)(c % ng);
        const int yi = adj_cell(i, t.x, N, ng), yj = adj_cell(j, t.y, N, ng), yk = adj_cell(k, t.z, N, ng);
        if (yi < 0 || yj < 0 || yk < 0) continue;
        const size_t y = ((size_t)yi * ng + yj) * ng + yk;
        acc = fmaf(recr[c], lr[y], acc);
        acc = fmaf(reci[c], li[y], acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) score[b] = v;
    }
}

// Score terms of one pose per warp for the detail output
// (src/docking.cpp:618-660, :733-812): the ligand cell l of the pose's
// voxel grid meets receptor cell l + tem - ng on each axis, with
// tem = (3 ng - t) mod 2 ng, over the same l, m, n ranges and in the same
// order as the reference, every product rounded before it is added (no
// FMA), so the float sums are the reference's.  terms[9 p ..]: direct sums of
// rPSC, ELEC and ACE products, then rPSC+, rPSC-, ELEC+, ELEC-, ACE+, ACE-.
// The sums are one sequential chain per pose, so one lane adds them; the
// warp's lanes load the next (l, m) row's z segment of the five grids
// (coalesced) while that lane adds the current row's terms from shared
// memory, so the loads' latency overlaps the chain instead of stalling it.
constexpr int kPoseTermWarps = 4;      // poses per CTA
constexpr int kPoseTermMaxNg = 256;    // longest z segment a row stages
__global__ void __launch_bounds__(32 * kPoseTermWarps)
    k_pose_terms(int ng, int n, const int4 *__restrict__ tem, const float *__restrict__ rec_r,
                 const float *__restrict__ rec_rpsc, const float *__restrict__ rec_i, const float *__restrict__ vr,
                 const float *__restrict__ vi, float *__restrict__ terms) {
    constexpr int PER = kPoseTermMaxNg / 32;
    __shared__ float stage[kPoseTermWarps][5][kPoseTermMaxNg];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = blockIdx.x * kPoseTermWarps + warp;
    if (p >= n) return;   // whole warps only
    const size_t ng2 = (size_t)ng * ng, ng3 = ng2 * ng;
    const int4 tc = tem[p];
    const int la = tc.x < ng ? ng - tc.x : 0, lb = tc.x < ng ? ng : 2 * ng - tc.x;
    const int ma = tc.y < ng ? ng - tc.y : 0, mb = tc.y < ng ? ng : 2 * ng - tc.y;
    const int na = tc.z < ng ? ng - tc.z : 0, nb = tc.z < ng ? ng : 2 * ng - tc.z;
    const int len = nb - na, per_l = mb - ma;
    const int rows = (len > 0 && per_l > 0 && lb > la) ? (lb - la) * per_l : 0;
    const float *lr = vr + (size_t)p * ng3, *li = vi + (size_t)p * ng3;
    float (*st)[kPoseTermMaxNg] = stage[warp];
    float nx[5][PER];
    // row r = (l, m) in the reference's order: l outer, m inner
    auto fetch = [&](int r) {
        const int l = la + r / per_l, m = ma + r % per_l;
        const size_t rz0 = ng2 * (size_t)(l + tc.x - ng) + (size_t)ng * (m + tc.y - ng) + (size_t)(tc.z + na - ng);
        const size_t lz0 = ng2 * (size_t)l + (size_t)ng * m + na;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int k = lane + 32 * j;
            if (k < len) {
                nx[0][j] = __ldg(&rec_rpsc[rz0 + k]);
                nx[1][j] = __ldg(&rec_r[rz0 + k]);
                nx[2][j] = __ldg(&rec_i[rz0 + k]);
                nx[3][j] = __ldg(&lr[lz0 + k]);
                nx[4][j] = __ldg(&li[lz0 + k]);
            }
        }
    };
    auto park = [&]() {
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int k = lane + 32 * j;
            if (k < len)
#pragma unroll
                for (int a = 0; a < 5; ++a) st[a][k] = nx[a][j];
        }
    };
    float s_rpsc = 0.f, s_elec = 0.f, s_ace = 0.f;
    float rp = 0.f, rm = 0.f, ep = 0.f, em = 0.f, ap = 0.f, am = 0.f;
    if (rows > 0) {
        fetch(0);
        park();
        __syncwarp();
    }
    for (int r = 0; r < rows; ++r) {
        if (r + 1 < rows) fetch(r + 1);
        if (lane == 0) {
            // the signed sums take each term through a select, not a branch:
            // the same additions in the same order
#pragma unroll 4
            for (int k = 0; k < len; ++k) {
                const float a = st[0][k], b = st[1][k], c = st[2][k];
                const float x = st[3][k], y = st[4][k];
                const float rpsc = __fmul_rn(a, x);
                const float elec = __fmul_rn(c, y);
                const float ace = __fmul_rn(__fsub_rn(b, a), x);
                s_rpsc = __fadd_rn(s_rpsc, rpsc);
                s_elec = __fadd_rn(s_elec, elec);
                s_ace = __fadd_rn(s_ace, ace);
                rm = rpsc < 0.f ? __fadd_rn(rm, rpsc) : rm;
                rp = rpsc > 0.f ? __fadd_rn(rp, rpsc) : rp;
                em = elec < 0.f ? __fadd_rn(em, elec) : em;
                ep = elec > 0.f ? __fadd_rn(ep, elec) : ep;
                am = ace < 0.f ? __fadd_rn(am, ace) : am;
                ap = ace > 0.f ? __fadd_rn(ap, ace) : ap;
            }
        }
        __syncwarp();
        if (r + 1 < rows) park();
        __syncwarp();
    }
    if (lane == 0) {
        float *o = terms + 9 * (size_t)p;
        o[0] = s_rpsc;
        o[1] = s_elec;
        o[2] = s_ace;
        o[3] = rp;
        o[4] = rm;
        o[5] = ep;
        o[6] = em;
        o[7] = ap;
        o[8] = am;
    }
}

}  // namespace mdb
