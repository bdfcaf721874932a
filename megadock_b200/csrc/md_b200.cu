// Device context and the device half of the C ABI (include/md_b200.h).
//
// Replaces FFTProcess's GPU members (src/fft_process.cpp:79-209 allocation,
// :212-303 receptor FFT, :502-656 per-rotation pipeline, :660-807 ligand
// voxelization and upload).  Differences by design:
//   - one context per device, explicit stream, no cudaDeviceSynchronize inside
//     the pipeline; a call returns after its own copies complete;
//   - no cuFFT: every transform is the project's fused FFT (dock_kernels.cuh);
//   - the batched form is one captured CUDA graph over the whole rotation
//     range, its launch groups alternating between two work sets on two
//     capture streams so that consecutive groups overlap on the GPU;
//   - errors are returned as status codes with a message, never exit().
#include "context.cuh"
#include "adjoint_kernels.cuh"
#include "receptor_kernels.cuh"

#include <atomic>

namespace {

// md_dock_pairs graphs kept per runner context before the cache is emptied
constexpr size_t kMaxPairGraphs = 32;

bool size_supported(int N) { return sized_ops(N) != nullptr; }

cudaError_t set_attrs(int N) {
    const SizedOps *o = sized_ops(N);
    return o ? o->set_attrs() : cudaErrorInvalidValue;
}

void launch_receptor(md_ctx *c, const float *r, const float *i) { sized_ops(c->N)->receptor(c, r, i); }

void launch_voxel_chunk(md_ctx *c, const float *rot, int nb, float *vr, float *vi) {
    sized_ops(c->N)->voxel_chunk(c, rot, nb, vr, vi);
}

void launch_voxels(md_ctx *c, const float *rot, float *vr, float *vi) { sized_ops(c->N)->voxels(c, rot, vr, vi); }

void launch_dock_ws(md_ctx *c, const WorkSet &w, cudaStream_t s, const float *rot, int nb, int rot0, int t,
                    DevPose *pose, cudaEvent_t *ev = nullptr) {
    sized_ops(c->N)->dock(c, w, s, rot, nb, rot0, t, pose, ev);
}

void launch_dock(md_ctx *c, int lane, cudaStream_t s, const float *rot, int nb, int rot0, int t, DevPose *pose,
                 cudaEvent_t *ev = nullptr) {
    launch_dock_ws(c, c->ws[lane], s, rot, nb, rot0, t, pose, ev);
}

void free_graphs(md_ctx *c) {
    ++c->gen;   // graphs of md_dock_pairs that captured this context's arguments no longer match
    for (auto &kv : c->graphs) cudaGraphExecDestroy(kv.second);
    c->graphs.clear();
    for (auto &kv : c->pair_graphs) cudaGraphExecDestroy(kv.second);
    c->pair_graphs.clear();
}

void release_work(md_ctx *c) {
    free_graphs(c);
    for (auto &w : c->ws) w.release();
    cudaFree(c->d_scratch);
    c->d_scratch = nullptr;
    c->scratch_cap = 0;
    c->cap = c->cap_t = c->cap_na = 0;
    c->sets = 0;
    c->have = WorkSet::Sizes{};
}

// At least `nsets` work sets holding at least `z` bytes per buffer (only the
// batched graph with two launch groups in flight and the pairs runner use the
// second set, so one launch group in flight holds one set on the device).
int ensure_bytes(md_ctx *ctx, const WorkSet::Sizes &z, int nsets) {
    bool ok = ctx->sets >= nsets;
    for (int k = 0; k < WorkSet::kBufs; ++k) ok = ok && z.b[k] <= ctx->have.b[k];
    if (ok) return MD_OK;
    WorkSet::Sizes m = ctx->have;
    for (int k = 0; k < WorkSet::kBufs; ++k) m.b[k] = std::max(m.b[k], z.b[k]);
    const int cap = ctx->cap, t = ctx->cap_t, na = ctx->cap_na;
    release_work(ctx);
    for (int k = 0; k < nsets; ++k) MD_CUDA(ctx->ws[k].allocate(m));
    ctx->sets = nsets;
    ctx->have = m;
    ctx->cap = cap;
    ctx->cap_t = t;
    ctx->cap_na = na;
    return MD_OK;
}

// `nsets` work sets for launch groups of `cap` rotations with t poses each.
int ensure_work(md_ctx *ctx, int cap, int t, int nsets = 1) {
    if (cap <= ctx->cap && t <= ctx->cap_t && ctx->na <= ctx->cap_na && nsets <= ctx->sets) return MD_OK;
    cap = std::max({cap, ctx->cap, 1});
    t = std::max({t, ctx->cap_t, 1});
    const int na = std::max({ctx->na, ctx->cap_na, 1});
    int rc = ensure_bytes(ctx, WorkSet::need(cap, ctx->N, t, na), nsets);
    if (rc) return rc;
    ctx->cap = cap;
    ctx->cap_t = t;
    ctx->cap_na = na;
    return MD_OK;
}

// Device scratch of the calls outside the docking graph (adjoint, pose
// scores, pose terms): n sub-buffers of sz[k] bytes, 256-byte aligned, carved
// from one context buffer that only grows, so repeated calls allocate nothing.
int carve_scratch(md_ctx *ctx, const size_t *sz, int n, char **out) {
    size_t off[16], total = 0;
    if (n > 16) return MD_ERR_ARG;
    for (int k = 0; k < n; ++k) {
        off[k] = total;
        total += (sz[k] + 255) & ~size_t(255);
    }
    if (total > ctx->scratch_cap) {
        MD_CUDA(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->d_scratch);
        ctx->d_scratch = nullptr;
        ctx->scratch_cap = 0;
        MD_CUDA(cudaMalloc(&ctx->d_scratch, total));
        ctx->scratch_cap = total;
    }
    for (int k = 0; k < n; ++k) out[k] = ctx->d_scratch + off[k];
    return MD_OK;
}

int check_ready(md_ctx *ctx) {
    if (!ctx->N) {
        ctx->err = "md_set_grid has not been called";
        return MD_ERR_STATE;
    }
    if (!ctx->have_receptor) {
        ctx->err = "md_receptor_fft has not been called";
        return MD_ERR_STATE;
    }
    if (!ctx->have_ligand) {
        ctx->err = "md_ligand_data has not been called";
        return MD_ERR_STATE;
    }
    return MD_OK;
}

// The rotation loop of one md_dock call on device buffers.
int run_dock(md_ctx *ctx, const float *d_rot, int first_rot, int n_rot, int t, DevPose *d_pose) {
    const int B = std::max(1, std::min(ctx->batch, n_rot));
    int rc = ensure_work(ctx, B, t, B == 1 ? 1 : ctx->lanes);
    if (rc) return rc;
    if (B == 1) {
        // plain form: one rotation per fused pipeline, launched back to back
        for (int r = 0; r < n_rot; ++r)
            launch_dock(ctx, 0, ctx->stream, d_rot + 9 * (size_t)r, 1, first_rot + r, t, d_pose + (size_t)r * t);
        MD_CUDA(cudaGetLastError());
        return MD_OK;
    }
    // batched form: the whole rotation loop as one captured CUDA graph; with
    // two lanes the launch groups alternate between the two work sets and the
    // two capture streams, with one they run back to back on one stream
    auto key = std::make_tuple(first_rot, n_rot, t, B, d_rot, d_pose);
    auto it = ctx->graphs.find(key);
    if (it == ctx->graphs.end()) {
        cudaGraph_t g;
        MD_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        cudaEventRecord(ctx->fork, ctx->stream);
        cudaStreamWaitEvent(ctx->side, ctx->fork, 0);
        int group = 0;
        for (int r = 0; r < n_rot; r += B, ++group) {
            const int nb = std::min(B, n_rot - r);
            const int lane = group % ctx->lanes;
            launch_dock(ctx, lane, lane ? ctx->side : ctx->stream, d_rot + 9 * (size_t)r, nb, first_rot + r, t,
                        d_pose + (size_t)r * t);
        }
        cudaEventRecord(ctx->join, ctx->side);
        cudaStreamWaitEvent(ctx->stream, ctx->join, 0);
        cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
        if (ce != cudaSuccess) {
            ctx->err = std::string("graph capture: ") + cudaGetErrorString(ce);
            return MD_ERR_CUDA;
        }
        cudaGraphExec_t ex;
        ce = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) {
            ctx->err = std::string("graph instantiate: ") + cudaGetErrorString(ce);
            return MD_ERR_CUDA;
        }
        it = ctx->graphs.emplace(key, ex).first;
    }
    MD_CUDA(cudaGraphLaunch(it->second, ctx->stream));
    return MD_OK;
}

}  // namespace

extern "C" {

int md_fft_size_supported(int nf1) { return size_supported(nf1) ? 1 : 0; }

int md_ctx_create(int device, md_ctx **out) {
    if (!out) return MD_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return MD_ERR_CUDA;
    if (device < 0 || device >= n) return MD_ERR_ARG;
    static std::atomic<uint64_t> next_uid{1};
    md_ctx *ctx = new md_ctx;
    ctx->device = device;
    ctx->uid = next_uid.fetch_add(1);
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->join, cudaEventDisableTiming) != cudaSuccess) {
        delete ctx;
        return MD_ERR_CUDA;
    }
    ctx->stream = ctx->own;
    *out = ctx;
    return MD_OK;
}

void md_ctx_destroy(md_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamSynchronize(ctx->side);
    release_work(ctx);
    cudaFree(ctx->d_gc);
    cudaFree(ctx->d_tw);
    cudaFree(ctx->d_Rh);
    cudaFree(ctx->d_recv);
    cudaFree(ctx->d_atom);
    cudaFree(ctx->d_rad2);
    cudaFree(ctx->d_rot);
    cudaFree(ctx->d_pose);
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    if (ctx->join) cudaEventDestroy(ctx->join);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
}

const char *md_last_error(const md_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int md_set_stream(md_ctx *ctx, void *stream) {
    if (!ctx) return MD_ERR_ARG;
    free_graphs(ctx);
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own;
    return MD_OK;
}

int md_set_grid(md_ctx *ctx, int nf1, float grid_width, const float *grid_coord) {
    if (!ctx || !grid_coord || !(grid_width > 0.f)) return MD_ERR_ARG;
    if (!size_supported(nf1)) {
        ctx->err = "FFT size " + std::to_string(nf1) +
                   " has no built kernel set (built: the default grid table's sizes up to 512; -F picks one)";
        return MD_ERR_SIZE;
    }
    MD_CUDA(cudaSetDevice(ctx->device));
    MD_CUDA(set_attrs(nf1));
    if (ctx->N != nf1) {
        release_work(ctx);
        cudaFree(ctx->d_gc);
        cudaFree(ctx->d_tw);
        cudaFree(ctx->d_Rh);
        cudaFree(ctx->d_recv);
        ctx->d_gc = nullptr;
        ctx->d_tw = nullptr;
        ctx->d_Rh = nullptr;
        ctx->d_recv = nullptr;
        ctx->have_receptor = false;
        const size_t N = nf1;
        MD_CUDA(cudaMalloc(&ctx->d_gc, sizeof(float) * N / 2));
        MD_CUDA(cudaMalloc(&ctx->d_tw, sizeof(float2) * N));
        MD_CUDA(cudaMalloc(&ctx->d_Rh, sizeof(float2) * N * N * N));
        MD_CUDA(cudaMalloc(&ctx->d_recv, sizeof(float) * 2 * (N / 2) * (N / 2) * (N / 2)));
        std::vector<float2> tw(N);
        for (size_t j = 0; j < N; ++j) {
            const double a = -2.0 * M_PI * (double)j / (double)N;
            tw[j] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        MD_CUDA(cudaMemcpyAsync(ctx->d_tw, tw.data(), sizeof(float2) * N, cudaMemcpyHostToDevice, ctx->stream));
        MD_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->N = nf1;
        ctx->ng = nf1 / 2;
    }
    if (ctx->gw != grid_width) free_graphs(ctx);   // the grid width is a kernel argument
    ctx->gw = grid_width;
    MD_CUDA(cudaMemcpyAsync(ctx->d_gc, grid_coord, sizeof(float) * ctx->ng, cudaMemcpyHostToDevice, ctx->stream));
    MD_CUDA(cudaStreamSynchronize(ctx->stream));
    return MD_OK;
}

int md_receptor_fft(md_ctx *ctx, const float *grid_r, const float *grid_i) {
    if (!ctx || !grid_r || !grid_i) return MD_ERR_ARG;
    if (!ctx->N) {
        ctx->err = "md_set_grid has not been called";
        return MD_ERR_STATE;
    }
    MD_CUDA(cudaSetDevice(ctx->device));
    int rc = ensure_work(ctx, std::max(1, ctx->batch), 1);
    if (rc) return rc;
    const size_t ng3 = (size_t)ctx->ng * ctx->ng * ctx->ng;
    float *d_r = ctx->d_recv, *d_i = ctx->d_recv + ng3;
    MD_CUDA(cudaMemcpyAsync(d_r, grid_r, sizeof(float) * ng3, cudaMemcpyHostToDevice, ctx->stream));
    MD_CUDA(cudaMemcpyAsync(d_i, grid_i, sizeof(float) * ng3, cudaMemcpyHostToDevice, ctx->stream));
    launch_receptor(ctx, d_r, d_i);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        ctx->err = std::string("receptor FFT: ") + cudaGetErrorString(e);
        return MD_ERR_CUDA;
    }
    ctx->have_receptor = true;
    return MD_OK;
}

int md_receptor_build(md_ctx *ctx, int na, const float *xyz_centred, const float *radius, const float *charge,
                      const float *ace, float rec_core, float ace_ratio, float elec_ratio, int make_receptor,
                      float *grid_r, float *grid_i) {
    if (!ctx || na < 1 || !xyz_centred || !radius || !charge || !ace) return MD_ERR_ARG;
    if (!ctx->N) {
        ctx->err = "md_set_grid has not been called";
        return MD_ERR_STATE;
    }
    const int ng = ctx->ng;
    if (ng > kRecMaxNg) {
        ctx->err = "receptor grids on the device are built for ng1 <= " + std::to_string(kRecMaxNg);
        return MD_ERR_SIZE;
    }
    MD_CUDA(cudaSetDevice(ctx->device));
    if (make_receptor) {
        int rc = ensure_work(ctx, std::max(1, ctx->batch), 1);
        if (rc) return rc;
    }
    const size_t ng3 = (size_t)ng * ng * ng;
    const float open_space = -7777.0f;
    // host copies of the two grid-coordinate values the reference reads
    std::vector<float> gc(ng);
    MD_CUDA(cudaMemcpy(gc.data(), ctx->d_gc, sizeof(float) * ng, cudaMemcpyDeviceToHost));
    RecParams P;
    P.ng = ng;
    P.na = na;
    P.gw = ctx->gw;
    P.width = gc[1] - gc[0];
    P.eps_core = rec_core;
    P.e_ratio = elec_ratio;
    P.cpg = -1 * P.width * 80.0f / (-2800.0f * elec_ratio);
    P.ace_ratio = (double)ace_ratio;
    P.reach_core = (int)((2.4 + ctx->gw - 0.01) / ctx->gw);
    P.reach_shell = (int)((12 + ctx->gw - 0.01) / ctx->gw);
    float *d_xyz = nullptr, *d_rad = nullptr, *d_q = nullptr, *d_ace = nullptr, *d_grid = nullptr;
    RecAtom *d_atoms = nullptr;
    int *d_cnt = nullptr, *d_start = nullptr, *d_list = nullptr;
    void *d_masks = nullptr;   // sweep row masks above ng = kRecSmemNg
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t x) {
        if (e == cudaSuccess) e = x;
    };
    auto cleanup = [&]() {
        cudaFree(d_xyz);
        cudaFree(d_rad);
        cudaFree(d_q);
        cudaFree(d_ace);
        cudaFree(d_atoms);
        cudaFree(d_cnt);
        cudaFree(d_start);
        cudaFree(d_list);
        cudaFree(d_masks);
        if (!make_receptor) cudaFree(d_grid);
    };
    cudaStream_t s = ctx->stream;
    step(cudaMalloc(&d_xyz, sizeof(float) * 3 * na));
    step(cudaMalloc(&d_rad, sizeof(float) * na));
    step(cudaMalloc(&d_q, sizeof(float) * na));
    step(cudaMalloc(&d_ace, sizeof(float) * na));
    step(cudaMalloc(&d_atoms, sizeof(RecAtom) * na));
    step(cudaMalloc(&d_cnt, sizeof(int) * (ng * ng + 1)));
    step(cudaMalloc(&d_start, sizeof(int) * (ng * ng + 1)));
    if (make_receptor) d_grid = ctx->d_recv;
    else step(cudaMalloc(&d_grid, sizeof(float) * 2 * ng3));
    if (e != cudaSuccess) {
        cleanup();
        ctx->err = std::string("receptor grids: ") + cudaGetErrorString(e);
        return MD_ERR_CUDA;
    }
    float *d_r = d_grid, *d_i = d_grid + ng3;
    step(cudaMemcpyAsync(d_xyz, xyz_centred, sizeof(float) * 3 * na, cudaMemcpyHostToDevice, s));
    step(cudaMemcpyAsync(d_rad, radius, sizeof(float) * na, cudaMemcpyHostToDevice, s));
    step(cudaMemcpyAsync(d_q, charge, sizeof(float) * na, cudaMemcpyHostToDevice, s));
    step(cudaMemcpyAsync(d_ace, ace, sizeof(float) * na, cudaMemcpyHostToDevice, s));
    step(cudaMemsetAsync(d_r, 0, sizeof(float) * ng3, s));
    const int rows = ng * ng;
    // the two propagation sweeps: row masks of ceil(ng / 64) words, in shared
    // memory up to ng = kRecSmemNg, else in a global buffer
    auto sweep = [&]() {
        if (ng <= kRecSmemNg) {
            const size_t smem = sizeof(RowMask<2>) * rows;
            step(cudaFuncSetAttribute(k_rec_sweep<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(RowMask<2>) * kRecSmemNg * kRecSmemNg)));
            for (int k = 0; k < 2 && e == cudaSuccess; ++k)
                k_rec_sweep<2, false><<<1, 1024, smem, s>>>(P, d_r, open_space, nullptr);
        } else if (ng <= 192) {
            step(cudaMalloc(&d_masks, sizeof(RowMask<3>) * rows));
            for (int k = 0; k < 2 && e == cudaSuccess; ++k)
                k_rec_sweep<3, true><<<1, 1024, 0, s>>>(P, d_r, open_space, static_cast<RowMask<3> *>(d_masks));
        } else {
            step(cudaMalloc(&d_masks, sizeof(RowMask<4>) * rows));
            for (int k = 0; k < 2 && e == cudaSuccess; ++k)
                k_rec_sweep<4, true><<<1, 1024, 0, s>>>(P, d_r, open_space, static_cast<RowMask<4> *>(d_masks));
        }
    };
    const int cells_blocks = (int)((ng3 + 255) / 256);
    std::vector<int> cnt(rows + 1), start(rows + 1);
    auto scan = [&](int n) {   // counts -> starts on the host (n + 1 entries)
        step(cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
        step(cudaStreamSynchronize(s));
        start[0] = 0;
        for (int r = 0; r < n; ++r) start[r + 1] = start[r] + cnt[r];
        step(cudaMemcpyAsync(d_start, start.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
        return start[n];
    };
    if (e == cudaSuccess) {
        k_rec_prep<<<(na + 255) / 256, 256, 0, s>>>(P, d_xyz, d_rad, d_q, d_ace, d_atoms);
        k_rec_core<<<na, 128, 0, s>>>(P, d_atoms, ctx->d_gc, d_r);
        k_rec_rays<<<(3 * rows + 255) / 256, 256, 0, s>>>(P, d_r, open_space);
        sweep();
        k_rec_final<<<cells_blocks, 256, 0, s>>>(P, d_r, open_space);
        // surface shell over per-row atom lists
        k_rec_rows<<<(rows + 3) / 4, 128, 0, s>>>(P, d_atoms, ctx->d_gc, d_cnt, nullptr, nullptr);
        const int nlist = scan(rows);
        step(cudaMalloc(&d_list, sizeof(int) * std::max(1, nlist)));
        if (e == cudaSuccess) {
            k_rec_rows<<<(rows + 3) / 4, 128, 0, s>>>(P, d_atoms, ctx->d_gc, d_cnt, d_start, d_list);
            k_rec_shell<<<cells_blocks, 256, 0, s>>>(P, d_atoms, ctx->d_gc, d_start, d_list, d_r);
            step(cudaGetLastError());
            step(cudaStreamSynchronize(s));
            cudaFree(d_list);
            d_list = nullptr;
        }
        // electrostatics over per-plane charged-atom lists
        if (e == cudaSuccess) {
            k_rec_planes<<<(ng + 3) / 4, 128, 0, s>>>(P, d_atoms, d_cnt, nullptr, nullptr);
            const int nplane = scan(ng);
            step(cudaMalloc(&d_list, sizeof(int) * std::max(1, nplane)));
        }
        if (e == cudaSuccess) {
            k_rec_planes<<<(ng + 3) / 4, 128, 0, s>>>(P, d_atoms, d_cnt, d_start, d_list);
            k_rec_elec<<<cells_blocks, 256, 0, s>>>(P, d_atoms, ctx->d_gc, d_start, d_list, d_r, d_i);
            if (make_receptor) launch_receptor(ctx, d_r, d_i);
            step(cudaGetLastError());
        }
        if (grid_r) step(cudaMemcpyAsync(grid_r, d_r, sizeof(float) * ng3, cudaMemcpyDeviceToHost, s));
        if (grid_i) step(cudaMemcpyAsync(grid_i, d_i, sizeof(float) * ng3, cudaMemcpyDeviceToHost, s));
        step(cudaStreamSynchronize(s));
    }
    cleanup();
    if (e != cudaSuccess) {
        ctx->err = std::string("receptor grids: ") + cudaGetErrorString(e);
        return MD_ERR_CUDA;
    }
    if (make_receptor) ctx->have_receptor = true;
    return MD_OK;
}

int md_receptor_spectrum(md_ctx *ctx, float *re, float *im) {
    if (!ctx || !re || !im) return MD_ERR_ARG;
    if (!ctx->have_receptor) {
        ctx->err = "no receptor spectrum";
        return MD_ERR_STATE;
    }
    const size_t n3 = (size_t)ctx->N * ctx->N * ctx->N;
    std::vector<float2> h(n3);
    MD_CUDA(cudaMemcpyAsync(h.data(), ctx->d_Rh, sizeof(float2) * n3, cudaMemcpyDeviceToHost, ctx->stream));
    MD_CUDA(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < n3; ++i) {
        re[i] = h[i].x;
        im[i] = h[i].y;
    }
    return MD_OK;
}

int md_ligand_data(md_ctx *ctx, int na, const float *xyz, const float *radius, const float *charge,
                   float lig_core) {
    if (!ctx || na <= 0 || !xyz || !radius || !charge) return MD_ERR_ARG;
    if (na > kMaxLigAtoms) {
        ctx->err = "ligand has " + std::to_string(na) + " atoms; at most " + std::to_string(kMaxLigAtoms) +
                   " are supported";
        return MD_ERR_SIZE;
    }
    if (lig_core == 0.0f || lig_core == -8888.0f) {
        ctx->err = "ligand core value (-b) 0 or -8888 collides with the voxelizer's markers";
        return MD_ERR_ARG;
    }
    MD_CUDA(cudaSetDevice(ctx->device));
    std::vector<float4> atom(na);
    std::vector<float2> rad(na);
    for (int l = 0; l < na; ++l) {
        atom[l] = make_float4(xyz[3 * l], xyz[3 * l + 1], xyz[3 * l + 2], charge[l]);
        // Ligand::precalc (src/ligand.cpp:251-254): R*R*1.5 and R*R*1.0 in float
        const float r = radius[l];
        rad[l] = make_float2(r * r * 1.5f, r * r * 1.0f);
    }
    if (na > ctx->na_cap) {
        free_graphs(ctx);
        cudaFree(ctx->d_atom);
        cudaFree(ctx->d_rad2);
        ctx->d_atom = nullptr;
        ctx->d_rad2 = nullptr;
        ctx->na_cap = 0;
        MD_CUDA(cudaMalloc(&ctx->d_atom, sizeof(float4) * na));
        MD_CUDA(cudaMalloc(&ctx->d_rad2, sizeof(float2) * na));
        ctx->na_cap = na;
    }
    // captured graphs hold the atom count and core value as kernel arguments;
    // new coordinates in the same buffers keep them valid
    if (na != ctx->na || lig_core != ctx->delta) free_graphs(ctx);
    MD_CUDA(cudaMemcpyAsync(ctx->d_atom, atom.data(), sizeof(float4) * na, cudaMemcpyHostToDevice, ctx->stream));
    MD_CUDA(cudaMemcpyAsync(ctx->d_rad2, rad.data(), sizeof(float2) * na, cudaMemcpyHostToDevice, ctx->stream));
    MD_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->na = na;
    ctx->delta = lig_core;
    ctx->have_ligand = true;
    return MD_OK;
}

int md_set_batch(md_ctx *ctx, int b) {
    if (!ctx || b < 1) return MD_ERR_ARG;
    ctx->batch = b;
    return MD_OK;
}

int md_release_work(md_ctx *ctx) {
    if (!ctx) return MD_ERR_ARG;
    MD_CUDA(cudaSetDevice(ctx->device));
    MD_CUDA(cudaStreamSynchronize(ctx->stream));
    MD_CUDA(cudaStreamSynchronize(ctx->side));
    release_work(ctx);
    return MD_OK;
}

int md_set_lanes(md_ctx *ctx, int lanes) {
    if (!ctx || lanes < 1 || lanes > kLanes) return MD_ERR_ARG;
    if (lanes != ctx->lanes) {
        free_graphs(ctx);
        ctx->lanes = lanes;
    }
    return MD_OK;
}

int md_set_tile(md_ctx *ctx, int lines) {
    if (!ctx || (lines != 8 && lines != 16 && lines != 32)) return MD_ERR_ARG;
    if (lines != ctx->tile) {
        free_graphs(ctx);
        ctx->tile = lines;
    }
    return MD_OK;
}

int md_set_plan(md_ctx *ctx, int plan) {
    if (!ctx || plan < 0 || plan >= kC2RPlans) return MD_ERR_ARG;
    if (plan != ctx->plan) {
        free_graphs(ctx);   // captured launches name the kernels
        ctx->plan = plan;
    }
    return MD_OK;
}

int md_dock_device(md_ctx *ctx, const float *d_rot, int first_rot, int n_rot, int t, md_pose *d_out) {
    if (!ctx || !d_rot || !d_out || n_rot < 0 || t < 1) return MD_ERR_ARG;
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (n_rot == 0) return MD_OK;
    MD_CUDA(cudaSetDevice(ctx->device));
    return run_dock(ctx, d_rot, first_rot, n_rot, t, reinterpret_cast<DevPose *>(d_out));
}

int md_dock(md_ctx *ctx, const float *rotmat, int first_rot, int n_rot, int t, md_pose *out) {
    if (!ctx || !rotmat || !out || n_rot < 0 || t < 1) return MD_ERR_ARG;
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (n_rot == 0) return MD_OK;
    MD_CUDA(cudaSetDevice(ctx->device));
    if ((size_t)n_rot * 9 > ctx->rot_cap) {
        free_graphs(ctx);
        cudaFree(ctx->d_rot);
        ctx->d_rot = nullptr;
        ctx->rot_cap = 0;
        MD_CUDA(cudaMalloc(&ctx->d_rot, sizeof(float) * 9 * n_rot));
        ctx->rot_cap = (size_t)n_rot * 9;
    }
    if ((size_t)n_rot * t > ctx->pose_cap) {
        free_graphs(ctx);
        cudaFree(ctx->d_pose);
        ctx->d_pose = nullptr;
        ctx->pose_cap = 0;
        MD_CUDA(cudaMalloc(&ctx->d_pose, sizeof(DevPose) * n_rot * t));
        ctx->pose_cap = (size_t)n_rot * t;
    }
    MD_CUDA(cudaMemcpyAsync(ctx->d_rot, rotmat, sizeof(float) * 9 * n_rot, cudaMemcpyHostToDevice, ctx->stream));
    rc = run_dock(ctx, ctx->d_rot, first_rot, n_rot, t, ctx->d_pose);
    if (rc) return rc;
    MD_CUDA(cudaMemcpyAsync(out, ctx->d_pose, sizeof(DevPose) * n_rot * t, cudaMemcpyDeviceToHost, ctx->stream));
    MD_CUDA(cudaStreamSynchronize(ctx->stream));
    return MD_OK;
}

int md_dock_profile(md_ctx *ctx, const float *d_rot, int first_rot, int n_rot, int t, md_pose *d_out,
                    float *stage_ms, int *launches) {
    if (!ctx || !d_rot || !d_out || !stage_ms || n_rot < 1 || t < 1) return MD_ERR_ARG;
    int rc = check_ready(ctx);
    if (rc) return rc;
    MD_CUDA(cudaSetDevice(ctx->device));
    const int B = std::max(1, std::min(ctx->batch, n_rot));
    if ((rc = ensure_work(ctx, B, t))) return rc;
    cudaEvent_t ev[6];
    for (auto &e : ev) MD_CUDA(cudaEventCreate(&e));
    double acc[5] = {0, 0, 0, 0, 0};
    int nl = 0;
    // atom prep, marks, voxelizer, forward planes, x lines, one top-t pass per
    // T poses, merge
    const int T = t == 1 ? 1 : (t <= 4 ? 4 : 16);
    const int per_group = 6 + (t + T - 1) / T;
    for (int r = 0; r < n_rot; r += B) {
        const int nb = std::min(B, n_rot - r);
        MD_CUDA(cudaEventRecord(ev[0], ctx->stream));
        launch_dock(ctx, 0, ctx->stream, d_rot + 9 * (size_t)r, nb, first_rot + r, t,
                    reinterpret_cast<DevPose *>(d_out) + (size_t)r * t, ev);
        nl += per_group;
        MD_CUDA(cudaEventSynchronize(ev[5]));
        for (int k = 0; k < 5; ++k) {
            float ms = 0.f;
            MD_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            acc[k] += ms;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    for (int k = 0; k < 5; ++k) stage_ms[k] = (float)acc[k];
    if (launches) *launches = nl;
    MD_CUDA(cudaGetLastError());
    return MD_OK;
}

int md_dock_pairs(md_ctx *runner, md_ctx *const *pairs, int npairs, const float *const *d_rotmat, const int *n_rot,
                  int t, md_pose *const *d_out) {
    md_ctx *ctx = runner;
    if (!ctx || !pairs || !d_rotmat || !n_rot || !d_out || npairs < 0 || t < 1) return MD_ERR_ARG;
    MD_CUDA(cudaSetDevice(ctx->device));
    // shared work sets: the largest launch group of any pair
    WorkSet::Sizes z{};
    std::vector<uintptr_t> key{(uintptr_t)npairs, (uintptr_t)t};
    for (int p = 0; p < npairs; ++p) {
        md_ctx *c = pairs[p];
        if (!c || !d_rotmat[p] || !d_out[p] || n_rot[p] < 0) return MD_ERR_ARG;
        if (c->device != ctx->device) {
            ctx->err = "md_dock_pairs: pair " + std::to_string(p) + " is on another device";
            return MD_ERR_ARG;
        }
        int rc = check_ready(c);
        if (rc) {
            ctx->err = "md_dock_pairs: pair " + std::to_string(p) + ": " + c->err;
            return rc;
        }
        MD_CUDA(set_attrs(c->N));
        const int B = std::max(1, std::min(c->batch, std::max(n_rot[p], 1)));
        const WorkSet::Sizes zp = WorkSet::need(B, c->N, t, std::max(c->na, 1));
        for (int k = 0; k < WorkSet::kBufs; ++k) z.b[k] = std::max(z.b[k], zp.b[k]);
        // the pair's (uid, gen) stands for every argument the capture takes
        // from it: grid width, core value, atom count, plan, tile and buffers
        key.insert(key.end(), {(uintptr_t)c->uid, (uintptr_t)c->gen, (uintptr_t)d_rotmat[p], (uintptr_t)n_rot[p],
                               (uintptr_t)d_out[p], (uintptr_t)B, (uintptr_t)c->na, (uintptr_t)c->N});
    }
    int rc = ensure_bytes(ctx, z, kLanes);
    if (rc) return rc;
    auto it = ctx->pair_graphs.find(key);
    if (it == ctx->pair_graphs.end()) {
        // keys of changed or destroyed pair contexts never match again: bound the cache
        if (ctx->pair_graphs.size() >= kMaxPairGraphs) {
            MD_CUDA(cudaStreamSynchronize(ctx->stream));
            for (auto &kv : ctx->pair_graphs) cudaGraphExecDestroy(kv.second);
            ctx->pair_graphs.clear();
        }
        cudaGraph_t g;
        MD_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        cudaEventRecord(ctx->fork, ctx->stream);
        cudaStreamWaitEvent(ctx->side, ctx->fork, 0);
        int group = 0;
        for (int p = 0; p < npairs; ++p) {
            md_ctx *c = pairs[p];
            const int B = std::max(1, std::min(c->batch, std::max(n_rot[p], 1)));
            DevPose *out = reinterpret_cast<DevPose *>(d_out[p]);
            for (int r = 0; r < n_rot[p]; r += B, ++group) {
                const int nb = std::min(B, n_rot[p] - r);
                const int lane = group % kLanes;
                launch_dock_ws(c, ctx->ws[lane], lane ? ctx->side : ctx->stream, d_rotmat[p] + 9 * (size_t)r, nb, r,
                               t, out + (size_t)r * t);
            }
        }
        cudaEventRecord(ctx->join, ctx->side);
        cudaStreamWaitEvent(ctx->stream, ctx->join, 0);
        cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
        if (ce != cudaSuccess) {
            ctx->err = std::string("graph capture: ") + cudaGetErrorString(ce);
            return MD_ERR_CUDA;
        }
        cudaGraphExec_t ex;
        ce = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) {
            ctx->err = std::string("graph instantiate: ") + cudaGetErrorString(ce);
            return MD_ERR_CUDA;
        }
        it = ctx->pair_graphs.emplace(key, ex).first;
    }
    MD_CUDA(cudaGraphLaunch(it->second, ctx->stream));
    return MD_OK;
}

namespace {

// Shared body of the adjoint entry points: per-pose rotation matrices (9 each),
// translations and weights dL/ds on the host; host outputs (any may be null).
int adjoint_core(md_ctx *ctx, const float *rotmat, int n, const int4 *shift, const float *w, float *d_rec_r,
                 float *d_rec_i, float *d_charge, const int *lig_sel, int n_lig, float *d_lig_r, float *d_lig_i,
                 float alpha, double *d_alpha) {
    MD_CUDA(cudaSetDevice(ctx->device));
    const int N = ctx->N, ng = ctx->ng;
    const size_t ng3 = (size_t)ng * ng * ng;
    const int B = std::max(1, std::min(ctx->batch, n));
    int rc = ensure_work(ctx, B, 1);
    if (rc) return rc;
    const size_t sz[8] = {sizeof(float) * 9 * n,       sizeof(float) * n,
                          sizeof(int4) * n,            sizeof(float) * 2 * ng3,
                          sizeof(float) * 2 * ng3 * B, sizeof(float) * std::max(ctx->na, 1),
                          sizeof(int) * std::max(n_lig, 1), sizeof(float) * 2 * ng3 * std::max(n_lig, 0)};
    char *p[8];
    if ((rc = carve_scratch(ctx, sz, 8, p))) return rc;
    float *d_rot = reinterpret_cast<float *>(p[0]), *d_w = reinterpret_cast<float *>(p[1]);
    int4 *d_shift = reinterpret_cast<int4 *>(p[2]);
    float *d_grad = reinterpret_cast<float *>(p[3]), *d_vox = reinterpret_cast<float *>(p[4]);
    float *d_dq = reinterpret_cast<float *>(p[5]);
    int *d_sel = reinterpret_cast<int *>(p[6]);
    float *d_lg = reinterpret_cast<float *>(p[7]);
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t x) {
        if (e == cudaSuccess) e = x;
    };
    cudaStream_t s = ctx->stream;
    step(cudaMemcpyAsync(d_rot, rotmat, sizeof(float) * 9 * n, cudaMemcpyHostToDevice, s));
    step(cudaMemcpyAsync(d_w, w, sizeof(float) * n, cudaMemcpyHostToDevice, s));
    step(cudaMemcpyAsync(d_shift, shift, sizeof(int4) * n, cudaMemcpyHostToDevice, s));
    step(cudaMemsetAsync(d_grad, 0, sizeof(float) * 2 * ng3, s));
    if (e != cudaSuccess) {
        ctx->err = std::string("adjoint: ") + cudaGetErrorString(e);
        return MD_ERR_CUDA;
    }
    const int thr = 256;
    const int blocks = (int)((ng3 + thr - 1) / thr);
    // receptor gradient: voxel grids of each chunk of poses, then the gather
    for (int r0 = 0; r0 < n; r0 += B) {
        const int nb = std::min(B, n - r0);
        launch_voxel_chunk(ctx, d_rot + 9 * (size_t)r0, nb, d_vox, d_vox + ng3 * B);
        k_adj_receptor<<<blocks, thr, 0, s>>>(N, ng, nb, d_vox, d_vox + ng3 * B, d_shift + r0, d_w + r0, d_grad,
                                              d_grad + ng3);
    }
    // charge gradient through the charge-cell assignment
    GridView G{ng, ctx->gw, (float)(ng * ctx->gw) / 2, ctx->d_gc, ctx->d_tw};
    LigandView L{ctx->na, ctx->d_atom, ctx->d_rad2, ctx->delta};
    k_adj_charge<<<(ctx->na + 3) / 4, 128, 0, s>>>(L, G, N, n, d_rot, d_shift, d_w, ctx->d_recv + ng3, d_dq);
    if (n_lig > 0) {
        step(cudaMemcpyAsync(d_sel, lig_sel, sizeof(int) * n_lig, cudaMemcpyHostToDevice, s));
        k_adj_ligand<<<dim3(blocks, n_lig), thr, 0, s>>>(N, ng, n_lig, d_sel, ctx->d_recv, ctx->d_recv + ng3,
                                                         d_shift, d_w, d_lg, d_lg + ng3 * n_lig);
    }
    step(cudaGetLastError());
    std::vector<float> gi(d_alpha ? ng3 : 0), ri(d_alpha ? ng3 : 0);
    if (d_rec_r) step(cudaMemcpyAsync(d_rec_r, d_grad, sizeof(float) * ng3, cudaMemcpyDeviceToHost, s));
    if (d_rec_i) step(cudaMemcpyAsync(d_rec_i, d_grad + ng3, sizeof(float) * ng3, cudaMemcpyDeviceToHost, s));
    if (d_alpha) {
        step(cudaMemcpyAsync(gi.data(), d_grad + ng3, sizeof(float) * ng3, cudaMemcpyDeviceToHost, s));
        step(cudaMemcpyAsync(ri.data(), ctx->d_recv + ng3, sizeof(float) * ng3, cudaMemcpyDeviceToHost, s));
    }
    if (d_charge) step(cudaMemcpyAsync(d_charge, d_dq, sizeof(float) * ctx->na, cudaMemcpyDeviceToHost, s));
    if (n_lig > 0) {
        step(cudaMemcpyAsync(d_lig_r, d_lg, sizeof(float) * ng3 * n_lig, cudaMemcpyDeviceToHost, s));
        step(cudaMemcpyAsync(d_lig_i, d_lg + ng3 * n_lig, sizeof(float) * ng3 * n_lig, cudaMemcpyDeviceToHost, s));
    }
    step(cudaStreamSynchronize(s));
    if (e != cudaSuccess) {
        ctx->err = std::string("adjoint: ") + cudaGetErrorString(e);
        return MD_ERR_CUDA;
    }
    if (d_alpha) {
        // the receptor's imaginary grid is alpha times a fixed-support unit grid
        double acc = 0.0;
        for (size_t x = 0; x < ng3; ++x) acc += (double)gi[x] * (double)ri[x];
        *d_alpha = alpha != 0.f ? acc / alpha : std::nan("");
    }
    return MD_OK;
}

int check_lig_sel(md_ctx *ctx, int n, const int *lig_sel, int n_lig, const float *a, const float *b) {
    if (n_lig < 0 || (n_lig > 0 && (!lig_sel || !a || !b))) return MD_ERR_ARG;
    for (int m = 0; m < n_lig; ++m)
        if (lig_sel[m] < 0 || lig_sel[m] >= n) {
            ctx->err = "ligand-grid selection outside the pose list";
            return MD_ERR_ARG;
        }
    return MD_OK;
}

}  // namespace

int md_adjoint_lse(md_ctx *ctx, const float *rotmat, int n_rot, const md_pose *top1, float temperature, float alpha,
                   double *loss, float *d_rec_r, float *d_rec_i, float *d_charge, double *d_alpha,
                   const int *lig_rot, int n_lig_rot, float *d_lig_r, float *d_lig_i) {
    if (!ctx || !rotmat || !top1 || n_rot < 1 || !(temperature > 0.f)) return MD_ERR_ARG;
    int rc = check_lig_sel(ctx, n_rot, lig_rot, n_lig_rot, d_lig_r, d_lig_i);
    if (rc) return rc;
    if ((rc = check_ready(ctx))) return rc;
    // loss and weights in double on the host: w_r = softmax(s_r / T); rotations
    // whose score was clamped to 0 (no positive cell) have no parameter gradient
    double smax = -1e300;
    for (int r = 0; r < n_rot; ++r) smax = std::max(smax, (double)top1[r].score);
    double z = 0.0;
    for (int r = 0; r < n_rot; ++r) z += std::exp(((double)top1[r].score - smax) / temperature);
    if (loss) *loss = smax + temperature * std::log(z);
    std::vector<float> w(n_rot);
    std::vector<int4> shift(n_rot);
    for (int r = 0; r < n_rot; ++r) {
        if (top1[r].i < 0 || top1[r].i >= ctx->N || top1[r].j < 0 || top1[r].j >= ctx->N || top1[r].k < 0 ||
            top1[r].k >= ctx->N) {
            ctx->err = "pose translation outside [0, nf1)";
            return MD_ERR_ARG;
        }
        const bool live = top1[r].score > 0.f;
        w[r] = live ? (float)(std::exp(((double)top1[r].score - smax) / temperature) / z) : 0.f;
        shift[r] = make_int4(top1[r].i, top1[r].j, top1[r].k, 0);
    }
    // only rotations with a nonzero float weight (or a requested ligand grid)
    // contribute: compact them, keeping their order
    std::vector<int> idx, remap(n_rot, -1);
    std::vector<char> want(n_rot, 0);
    for (int m = 0; m < n_lig_rot; ++m) want[lig_rot[m]] = 1;
    for (int r = 0; r < n_rot; ++r)
        if (w[r] != 0.f || want[r]) {
            remap[r] = (int)idx.size();
            idx.push_back(r);
        }
    if (idx.empty()) {   // no live rotation: every gradient is zero
        const size_t ng3 = (size_t)ctx->ng * ctx->ng * ctx->ng;
        if (d_rec_r) std::fill(d_rec_r, d_rec_r + ng3, 0.f);
        if (d_rec_i) std::fill(d_rec_i, d_rec_i + ng3, 0.f);
        if (d_charge) std::fill(d_charge, d_charge + ctx->na, 0.f);
        if (d_alpha) *d_alpha = 0.0;
        return MD_OK;
    }
    const int nc = (int)idx.size();
    std::vector<float> mc(9 * (size_t)nc), wc(nc);
    std::vector<int4> sc(nc);
    for (int c = 0; c < nc; ++c) {
        std::copy(rotmat + 9 * (size_t)idx[c], rotmat + 9 * (size_t)idx[c] + 9, mc.begin() + 9 * (size_t)c);
        wc[c] = w[idx[c]];
        sc[c] = shift[idx[c]];
    }
    std::vector<int> lc(n_lig_rot);
    for (int m = 0; m < n_lig_rot; ++m) lc[m] = remap[lig_rot[m]];
    return adjoint_core(ctx, mc.data(), nc, sc.data(), wc.data(), d_rec_r, d_rec_i, d_charge, lc.data(), n_lig_rot,
                        d_lig_r, d_lig_i, alpha, d_alpha);
}

int md_adjoint_poses(md_ctx *ctx, const float *rotmat, int n, const md_pose *poses, const float *dl_ds,
                     float *d_rec_r, float *d_rec_i, float *d_charge, const int *lig_pose, int n_lig,
                     float *d_lig_r, float *d_lig_i) {
    if (!ctx || !rotmat || !poses || !dl_ds || n < 1) return MD_ERR_ARG;
    int rc = check_lig_sel(ctx, n, lig_pose, n_lig, d_lig_r, d_lig_i);
    if (rc) return rc;
    if ((rc = check_ready(ctx))) return rc;
    std::vector<int4> shift(n);
    for (int r = 0; r < n; ++r) {
        if (poses[r].i < 0 || poses[r].i >= ctx->N || poses[r].j < 0 || poses[r].j >= ctx->N || poses[r].k < 0 ||
            poses[r].k >= ctx->N) {
            ctx->err = "pose translation outside [0, nf1)";
            return MD_ERR_ARG;
        }
        shift[r] = make_int4(poses[r].i, poses[r].j, poses[r].k, 0);
    }
    return adjoint_core(ctx, rotmat, n, shift.data(), dl_ds, d_rec_r, d_rec_i, d_charge, lig_pose, n_lig, d_lig_r,
                        d_lig_i, 0.f, nullptr);
}

int md_pose_scores(md_ctx *ctx, const float *rotmat, int n, const md_pose *poses, float *scores) {
    if (!ctx || !rotmat || !poses || !scores || n < 1) return MD_ERR_ARG;
    int rc = check_ready(ctx);
    if (rc) return rc;
    MD_CUDA(cudaSetDevice(ctx->device));
    const int N = ctx->N, ng = ctx->ng;
    const size_t ng3 = (size_t)ng * ng * ng;
    std::vector<int4> shift(n);
    for (int r = 0; r < n; ++r) {
        if (poses[r].i < 0 || poses[r].i >= N || poses[r].j < 0 || poses[r].j >= N || poses[r].k < 0 ||
            poses[r].k >= N) {
            ctx->err = "pose translation outside [0, nf1)";
            return MD_ERR_ARG;
        }
        shift[r] = make_int4(poses[r].i, poses[r].j, poses[r].k, 0);
    }
    const int B = std::max(1, std::min(ctx->batch, n));
    if ((rc = ensure_work(ctx, B, 1))) return rc;
    const size_t sz[4] = {sizeof(float) * 9 * n, sizeof(int4) * n, sizeof(float) * n, sizeof(float) * 2 * ng3 * B};
    char *p[4];
    if ((rc = carve_scratch(ctx, sz, 4, p))) return rc;
    float *d_rot = reinterpret_cast<float *>(p[0]), *d_sc = reinterpret_cast<float *>(p[2]);
    int4 *d_shift = reinterpret_cast<int4 *>(p[1]);
    float *d_vox = reinterpret_cast<float *>(p[3]);
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t x) {
        if (e == cudaSuccess) e = x;
    };
    cudaStream_t s = ctx->stream;
    step(cudaMemcpyAsync(d_rot, rotmat, sizeof(float) * 9 * n, cudaMemcpyHostToDevice, s));
    step(cudaMemcpyAsync(d_shift, shift.data(), sizeof(int4) * n, cudaMemcpyHostToDevice, s));
    if (e == cudaSuccess) {
        for (int r0 = 0; r0 < n; r0 += B) {
            const int nb = std::min(B, n - r0);
            launch_voxel_chunk(ctx, d_rot + 9 * (size_t)r0, nb, d_vox, d_vox + ng3 * B);
            k_pose_dot<<<nb, 512, 0, s>>>(N, ng, ctx->d_recv, ctx->d_recv + ng3, d_vox, d_vox + ng3 * B,
                                          d_shift + r0, d_sc + r0);
        }
        step(cudaGetLastError());
        step(cudaMemcpyAsync(scores, d_sc, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
        step(cudaStreamSynchronize(s));
    }
    if (e != cudaSuccess) {
        ctx->err = std::string("pose scores: ") + cudaGetErrorString(e);
        return MD_ERR_CUDA;
    }
    return MD_OK;
}

int md_pose_terms(md_ctx *ctx, const float *rec_rpsc, const float *rotmat, int n, const int *tem3, float *terms) {
    if (!ctx || !rec_rpsc || !rotmat || !tem3 || !terms || n < 1) return MD_ERR_ARG;
    int rc = check_ready(ctx);
    if (rc) return rc;
    const int ng = ctx->ng;
    for (int p = 0; p < 3 * n; ++p)
        if (tem3[p] < 0 || tem3[p] >= 2 * ng) {
            ctx->err = "pose offset outside [0, nf1)";
            return MD_ERR_ARG;
        }
    if (ng > kPoseTermMaxNg) {
        ctx->err = "pose terms: grid edge above " + std::to_string(kPoseTermMaxNg);
        return MD_ERR_SIZE;
    }
    MD_CUDA(cudaSetDevice(ctx->device));
    const size_t ng3 = (size_t)ng * ng * ng;
    // poses per launch: their voxel grids within about 1 GB
    const int P = (int)std::max<size_t>(1, std::min<size_t>((size_t)n, ((size_t)1 << 30) / (8 * ng3)));
    const int B = std::max(1, std::min(ctx->batch, P));
    if ((rc = ensure_work(ctx, B, 1))) return rc;
    float *d_rot = nullptr, *d_vox = nullptr, *d_terms = nullptr, *d_rpsc = nullptr;
    int4 *d_tem = nullptr;
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t x) {
        if (e == cudaSuccess) e = x;
    };
    std::vector<int4> tem(n);
    for (int p = 0; p < n; ++p) tem[p] = make_int4(tem3[3 * p], tem3[3 * p + 1], tem3[3 * p + 2], 0);
    step(cudaMalloc(&d_rot, sizeof(float) * 9 * n));
    step(cudaMalloc(&d_tem, sizeof(int4) * n));
    step(cudaMalloc(&d_terms, sizeof(float) * 9 * n));
    step(cudaMalloc(&d_rpsc, sizeof(float) * ng3));
    step(cudaMalloc(&d_vox, sizeof(float) * 2 * ng3 * P));
    cudaStream_t s = ctx->stream;
    step(cudaMemcpyAsync(d_rot, rotmat, sizeof(float) * 9 * n, cudaMemcpyHostToDevice, s));
    step(cudaMemcpyAsync(d_tem, tem.data(), sizeof(int4) * n, cudaMemcpyHostToDevice, s));
    step(cudaMemcpyAsync(d_rpsc, rec_rpsc, sizeof(float) * ng3, cudaMemcpyHostToDevice, s));
    if (e == cudaSuccess) {
        for (int p0 = 0; p0 < n; p0 += P) {
            const int np = std::min(P, n - p0);
            for (int b0 = 0; b0 < np; b0 += B) {
                const int nb = std::min(B, np - b0);
                // the chunk's grids at [b0, b0 + nb) of the P-pose buffers
                launch_voxel_chunk(ctx, d_rot + 9 * (size_t)(p0 + b0), nb, d_vox + ng3 * b0,
                                   d_vox + ng3 * ((size_t)P + b0));
            }
            k_pose_terms<<<(np + kPoseTermWarps - 1) / kPoseTermWarps, 32 * kPoseTermWarps, 0, s>>>(
                ng, np, d_tem + p0, ctx->d_recv, d_rpsc, ctx->d_recv + ng3, d_vox, d_vox + ng3 * P,
                d_terms + 9 * (size_t)p0);
        }
        step(cudaGetLastError());
        step(cudaMemcpyAsync(terms, d_terms, sizeof(float) * 9 * n, cudaMemcpyDeviceToHost, s));
        step(cudaStreamSynchronize(s));
    }
    cudaFree(d_rot);
    cudaFree(d_tem);
    cudaFree(d_terms);
    cudaFree(d_rpsc);
    cudaFree(d_vox);
    if (e != cudaSuccess) {
        ctx->err = std::string("pose terms: ") + cudaGetErrorString(e);
        return MD_ERR_CUDA;
    }
    return MD_OK;
}

int md_ligand_voxels(md_ctx *ctx, const float *rotmat9, float *grid_r, float *grid_i) {
    if (!ctx || !rotmat9 || !grid_r || !grid_i) return MD_ERR_ARG;
    if (!ctx->N || !ctx->have_ligand) {
        ctx->err = "grid and ligand must be set first";
        return MD_ERR_STATE;
    }
    MD_CUDA(cudaSetDevice(ctx->device));
    int rc = ensure_work(ctx, std::max(1, ctx->batch), 1);
    if (rc) return rc;
    const size_t ng3 = (size_t)ctx->ng * ctx->ng * ctx->ng;
    float *d = nullptr;
    MD_CUDA(cudaMalloc(&d, sizeof(float) * (ng3 * 2 + 9)));
    float *d_vr = d, *d_vi = d + ng3, *d_rot = d + 2 * ng3;
    cudaError_t e = cudaMemcpyAsync(d_rot, rotmat9, sizeof(float) * 9, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        launch_voxels(ctx, d_rot, d_vr, d_vi);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(grid_r, d_vr, sizeof(float) * ng3, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(grid_i, d_vi, sizeof(float) * ng3, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    if (e != cudaSuccess) {
        ctx->err = std::string("voxelization: ") + cudaGetErrorString(e);
        return MD_ERR_CUDA;
    }
    return MD_OK;
}

}  // extern "C"
