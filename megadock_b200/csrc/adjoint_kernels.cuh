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

// Score terms of one pose per thread for the detail output
// (src/docking.cpp:618-660, :733-812): the ligand cell l of the pose's
// voxel grid meets receptor cell l + tem - ng on each axis, with
// tem = (3 ng - t) mod 2 ng, over the same l, m, n ranges and in the same
// order as the reference, every product rounded before it is added (no
// FMA), so the float sums are the reference's.  terms[9 p ..]: direct sums of
// rPSC, ELEC and ACE products, then rPSC+, rPSC-, ELEC+, ELEC-, ACE+, ACE-.
__global__ void k_pose_terms(int ng, int n, const int4 *__restrict__ tem, const float *__restrict__ rec_r,
                             const float *__restrict__ rec_rpsc, const float *__restrict__ rec_i,
                             const float *__restrict__ vr, const float *__restrict__ vi, float *__restrict__ terms) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const size_t ng2 = (size_t)ng * ng, ng3 = ng2 * ng;
    const int4 tc = tem[p];
    const int la = tc.x < ng ? ng - tc.x : 0, lb = tc.x < ng ? ng : 2 * ng - tc.x;
    const int ma = tc.y < ng ? ng - tc.y : 0, mb = tc.y < ng ? ng : 2 * ng - tc.y;
    const int na = tc.z < ng ? ng - tc.z : 0, nb = tc.z < ng ? ng : 2 * ng - tc.z;
    const float *lr = vr + (size_t)p * ng3, *li = vi + (size_t)p * ng3;
    float s_rpsc = 0.f, s_elec = 0.f, s_ace = 0.f;
    float rp = 0.f, rm = 0.f, ep = 0.f, em = 0.f, ap = 0.f, am = 0.f;
    for (int l = la; l < lb; ++l) {
        const size_t rxc = ng2 * (size_t)(l + tc.x - ng), lxc = ng2 * (size_t)l;
        for (int m = ma; m < mb; ++m) {
            const size_t ryc = rxc + (size_t)ng * (m + tc.y - ng), lyc = lxc + (size_t)ng * m;
            // unrolled so that the loads of several cells are in flight
            // while the sums, whose order is fixed, run one cell at a time
#pragma unroll 8
            for (int k = na; k < nb; ++k) {
                const size_t rzc = ryc + (size_t)(tc.z + k - ng), lzc = lyc + k;
                const float a = __ldg(&rec_rpsc[rzc]), b = __ldg(&rec_r[rzc]), c = __ldg(&rec_i[rzc]);
                const float x = __ldg(&lr[lzc]), y = __ldg(&li[lzc]);
                const float rpsc = __fmul_rn(a, x);
                const float elec = __fmul_rn(c, y);
                const float ace = __fmul_rn(__fsub_rn(b, a), x);
                s_rpsc = __fadd_rn(s_rpsc, rpsc);
                s_elec = __fadd_rn(s_elec, elec);
                s_ace = __fadd_rn(s_ace, ace);
                if (rpsc < 0.f) rm = __fadd_rn(rm, rpsc);
                else if (rpsc > 0.f) rp = __fadd_rn(rp, rpsc);
                if (elec < 0.f) em = __fadd_rn(em, elec);
                else if (elec > 0.f) ep = __fadd_rn(ep, elec);
                if (ace < 0.f) am = __fadd_rn(am, ace);
                else if (ace > 0.f) ap = __fadd_rn(ap, ace);
            }
        }
    }
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

}  // namespace mdb
