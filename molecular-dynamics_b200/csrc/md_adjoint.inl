// Host orchestration of the trajectory adjoint (md_adjoint_* in include/md_b200.h). Included at the end of
// md_abi.cu. Kernels and the arithmetic are in md_adjoint.cuh.
//
// Forward: K velocity-Verlet steps from the initial state, recording U_k, W_k and KE_k, with a checkpoint of
// (positions, velocities, list reference positions) before every `every`-th step. Backward: segments in
// reverse; each is recomputed from its checkpoint (same bits: the list is rebuilt from the stored reference
// positions, and every rebuild decision repeats), keeping every state and the reference positions of every
// list built, then walked back step by step: the objective's terms at s_j, the second half kick's pass at r_j,
// the drift, the first half kick's pass at r_{j-1}.

#include <memory>

struct md_adjoint {
    int device = 0;
    cudaStream_t stream = nullptr;
    int n = 0;
    Box box{};
    double volume = 0.0;
    double eps = 1.0, sigma = 1.0, rc = 2.5, skin = 0.3, dt = 0.005;
    int steps = 0, every = 1;
    AdjConsts c{};
    double rl2 = 0.0, max_disp2 = 0.0, half_dt = 0.0;
    DevBuf<double4> pos, pos0, ref;
    DevBuf<double> vel, vel0, force, mass, u, w;
    CellGrid grid;
    int cap = 0;
    DevBuf<uint32_t> rows;
    DevBuf<int> counts, flags;
    DevBuf<double2> blocks;
    DevBuf<double> scal;  // [0..1] sum u, sum w; [2..3] kinetic (+ scratch); [4..5] running sums; [6..11] pass sums;
                          // [12..13] theta
    DevBuf<double> U, W, KE;
    std::vector<std::unique_ptr<DevBuf<double4>>> ck_pos, ck_ref;
    std::vector<std::unique_ptr<DevBuf<double>>> ck_vel;
    std::vector<std::unique_ptr<DevBuf<double4>>> seg_pos, gen_ref;
    std::vector<std::unique_ptr<DevBuf<double>>> seg_vel;
    std::vector<int> seg_gen;
    DevBuf<double> ar, av, wv, pe, ps, us, ws, ue, we;
    double meanU = 0.0, meanP = 0.0;
    bool forwarded = false;
    int rebuilds = 0;  // list builds of the last forward pass (the first included)
    int* h_flag = nullptr;
    uint64_t launches = 0;
    ~md_adjoint() {
        if (h_flag) cudaFreeHost(h_flag);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

constexpr int kS_UW = 0, kS_KE = 2, kS_RUN = 4, kS_PASS = 6, kS_THETA = 12;

md_status use_adjoint(md_adjoint* a) {
    g_launches = &a->launches;
    MD_CUDA(cudaSetDevice(a->device));
    return MD_OK;
}

md_status async_copy(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    MD_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st));
    return MD_OK;
}

void adj_constants(md_adjoint* a) {
    const LJ lj = lj_constants(a->eps, a->sigma, a->rc);
    a->c.box = a->box;
    a->c.sig2 = lj.sig2;
    a->c.eps24 = lj.eps24;
    a->c.eps4 = lj.eps4;
    a->c.shift = lj.shift;
    a->c.rc2 = lj.rc2;
    a->c.eps = a->eps;
    a->c.inv_sigma = 1.0 / a->sigma;
    const double sr6 = std::pow(a->sigma / a->rc, 6);
    const double sr12 = sr6 * sr6;
    a->c.shift_sigma = 4.0 * a->eps * (12.0 * sr12 - 6.0 * sr6) / a->sigma;  // d shift / d sigma
}

// The list at positions p (which become its reference positions): stable cell sort of indices, then full rows
md_status adj_build(md_adjoint* a, const double4* p) {
    cudaStream_t st = a->stream;
    const int n = a->n;
    MD_TRY(async_copy(a->ref.p, p, sizeof(double4) * n, st));
    CellGrid& g = a->grid;
    g.ncps = std::max(1, static_cast<int>(a->box.L / (a->rc + a->skin)));  // src/CellList.cpp:14
    g.ncells = g.ncps * g.ncps * g.ncps;
    const double inv_cell = g.ncps / a->box.L;
    MD_CUDA(g.cell_of.reserve(n));
    MD_CUDA(g.count.reserve(g.ncells));
    MD_CUDA(g.cursor.reserve(g.ncells));
    MD_CUDA(g.start.reserve(g.ncells + 1));
    MD_CUDA(g.bucket.reserve(n));
    MD_CUDA(g.order.reserve(n));
    MD_CUDA(g.tiles.reserve(scan_tiles_needed(g.ncells)));
    MD_CUDA(cudaMemsetAsync(g.count.p, 0, sizeof(int) * g.ncells, st));
    MD_CUDA(cudaMemsetAsync(g.cursor.p, 0, sizeof(int) * g.ncells, st));
    k_cell_assign<<<blocks_for(n, kThreads), kThreads, 0, st>>>(p, n, inv_cell, g.ncps, g.cell_of.p, g.count.p);
    MD_CHECK_LAUNCH();
    exclusive_scan<int, int>(g.count.p, g.ncells, g.start.p, g.tiles.p, st);
    MD_CHECK_SCAN();
    k_cell_scatter<<<blocks_for(n, kThreads), kThreads, 0, st>>>(g.cell_of.p, n, g.start.p, g.cursor.p, g.bucket.p);
    MD_CHECK_LAUNCH();
    k_cell_rank<<<blocks_for(static_cast<long long>(g.ncells) * 32, kThreads), kThreads, 0, st>>>(
        g.start.p, g.ncells, g.bucket.p, g.order.p);
    MD_CHECK_LAUNCH();
    for (int attempt = 0; attempt < 4; ++attempt) {
        MD_CUDA(a->rows.reserve(row_buffer_entries(n, a->cap)));
        MD_CUDA(cudaMemsetAsync(a->flags.p, 0, sizeof(int), st));
        k_adj_rows<<<blocks_for(n, 128), 128, 0, st>>>(p, n, a->box, a->rl2, g.ncps, g.cell_of.p, g.start.p, g.order.p,
                                                       a->cap, a->rows.p, a->counts.p, a->flags.p);
        MD_CHECK_LAUNCH();
        MD_CUDA(cudaMemcpyAsync(a->h_flag, a->flags.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        MD_CUDA(cudaStreamSynchronize(st));
        if (*a->h_flag <= a->cap) return MD_OK;
        a->cap = ((*a->h_flag + *a->h_flag / 4 + 16) + 7) & ~7;
        a->rows.release();
    }
    return fail(MD_ERR_CAPACITY, "neighbour row capacity could not be met");
}

md_status adj_forces(md_adjoint* a) {
    k_adj_forces<<<blocks_for(a->n, 128), 128, 0, a->stream>>>(a->pos.p, a->n, a->c, a->rows.p, a->cap, a->counts.p,
                                                               a->force.p, a->u.p, a->w.p);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

// Blocked sums of two per-particle arrays into out[0], out[1]
md_status adj_sum2(md_adjoint* a, const double* x, const double* y, double* out) {
    const int nb = (a->n + kChunk - 1) / kChunk;
    const size_t smem = 4 * kChunk * sizeof(double2);
    k_adj_blocks2<<<blocks_for(nb, 4), 128, smem, a->stream>>>(x, y, a->n, a->blocks.p, nb);
    MD_CHECK_LAUNCH();
    k_sum_blocks<<<1, 32, 0, a->stream>>>(a->blocks.p, nb, out);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

// One step (src/Integrator.cpp:18-30 without the reorder); *rebuilt says whether the list was rebuilt
md_status adj_step(md_adjoint* a, bool* rebuilt) {
    cudaStream_t st = a->stream;
    const int n = a->n;
    MD_CUDA(cudaMemsetAsync(a->flags.p + 1, 0, sizeof(int), st));
    k_kick_drift<<<blocks_for(n, kThreads), kThreads, 0, st>>>(a->pos.p, a->vel.p, a->force.p, a->mass.p, n, a->half_dt,
                                                                a->dt, a->box, a->ref.p, a->max_disp2, a->flags.p + 1);
    MD_CHECK_LAUNCH();
    MD_CUDA(cudaMemcpyAsync(a->h_flag, a->flags.p + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    MD_CUDA(cudaStreamSynchronize(st));
    *rebuilt = *a->h_flag != 0;
    if (*rebuilt) MD_TRY(adj_build(a, a->pos.p));
    MD_TRY(adj_forces(a));
    k_kick<<<blocks_for(n, kThreads), kThreads, 0, st>>>(a->vel.p, a->force.p, a->mass.p, n, a->half_dt);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

// A backward pass at positions p with the weights in a->wv
md_status adj_pass(md_adjoint* a, const double4* p, double aU, double aW, bool objective) {
    cudaStream_t st = a->stream;
    k_adj_pass<<<blocks_for(a->n, 128), 128, 0, st>>>(p, a->n, a->c, a->rows.p, a->cap, a->counts.p, a->wv.p, aU, aW,
                                                      a->ar.p, a->pe.p, a->ps.p, a->us.p, a->ws.p, a->ue.p, a->we.p);
    MD_CHECK_LAUNCH();
    double* sums = a->scal.p + kS_PASS;
    MD_TRY(adj_sum2(a, a->pe.p, a->ps.p, sums));
    if (objective) {
        MD_TRY(adj_sum2(a, a->us.p, a->ws.p, sums + 2));
        MD_TRY(adj_sum2(a, a->ue.p, a->we.p, sums + 4));
    }
    k_adj_theta<<<1, 1, 0, st>>>(sums, a->eps, aU, aW, objective, a->scal.p + kS_THETA);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

md_status adj_weights(md_adjoint* a) {
    k_adj_weights<<<blocks_for(3ll * a->n, kThreads), kThreads, 0, a->stream>>>(a->av.p, a->mass.p, a->n, a->half_dt,
                                                                               a->wv.p);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

template <typename T>
md_status keep(std::vector<std::unique_ptr<DevBuf<T>>>& v, size_t k, size_t count) {
    while (v.size() <= k) v.push_back(std::make_unique<DevBuf<T>>());
    MD_CUDA(v[k]->reserve(count));
    return MD_OK;
}

md_status adj_forward(md_adjoint* a) {
    cudaStream_t st = a->stream;
    const size_t n = a->n;
    MD_TRY(async_copy(a->pos.p, a->pos0.p, sizeof(double4) * n, st));
    MD_TRY(async_copy(a->vel.p, a->vel0.p, sizeof(double) * 3 * n, st));
    MD_TRY(adj_build(a, a->pos.p));
    a->rebuilds = 1;
    MD_TRY(adj_forces(a));
    MD_CUDA(cudaMemsetAsync(a->scal.p + kS_RUN, 0, 2 * sizeof(double), st));
    MD_CUDA(a->U.reserve(a->steps + 1));
    MD_CUDA(a->W.reserve(a->steps + 1));
    MD_CUDA(a->KE.reserve(a->steps + 1));
    const int nb = (a->n + kChunk - 1) / kChunk;
    for (int k = 1; k <= a->steps; ++k) {
        if ((k - 1) % a->every == 0) {
            const size_t c = (k - 1) / a->every;
            MD_TRY(keep(a->ck_pos, c, n));
            MD_TRY(keep(a->ck_ref, c, n));
            MD_TRY(keep(a->ck_vel, c, 3 * n));
            MD_TRY(async_copy(a->ck_pos[c]->p, a->pos.p, sizeof(double4) * n, st));
            MD_TRY(async_copy(a->ck_ref[c]->p, a->ref.p, sizeof(double4) * n, st));
            MD_TRY(async_copy(a->ck_vel[c]->p, a->vel.p, sizeof(double) * 3 * n, st));
        }
        bool rebuilt = false;
        MD_TRY(adj_step(a, &rebuilt));
        a->rebuilds += rebuilt ? 1 : 0;
        MD_TRY(adj_sum2(a, a->u.p, a->w.p, a->scal.p + kS_UW));
        const size_t smem = kEnergyWarps * kChunk * sizeof(double);
        k_kinetic_blocks<<<blocks_for(nb, kEnergyWarps), kEnergyWarps * 32, smem, st>>>(a->vel.p, a->mass.p, a->n,
                                                                                       a->blocks.p, nb);
        MD_CHECK_LAUNCH();
        k_sum_blocks<<<1, 32, 0, st>>>(a->blocks.p, nb, a->scal.p + kS_KE);
        MD_CHECK_LAUNCH();
        k_adj_record<<<1, 1, 0, st>>>(a->scal.p + kS_UW, a->scal.p + kS_KE, a->volume, k, a->U.p, a->W.p, a->KE.p,
                                      a->scal.p + kS_RUN);
        MD_CHECK_LAUNCH();
    }
    double run[2];
    MD_CUDA(cudaMemcpyAsync(run, a->scal.p + kS_RUN, sizeof(run), cudaMemcpyDeviceToHost, st));
    MD_CUDA(cudaStreamSynchronize(st));
    a->meanU = run[0] / a->steps;
    a->meanP = run[1] / a->steps;
    a->forwarded = true;
    return MD_OK;
}

md_status adj_backward(md_adjoint* a, double gU, double gP) {
    cudaStream_t st = a->stream;
    const size_t n = a->n;
    const double aU = gU / a->steps;
    const double aW = gP / (3.0 * a->volume * a->steps);
    const double aK = 2.0 * aW;
    const bool objective = aU != 0.0 || aW != 0.0;
    MD_CUDA(cudaMemsetAsync(a->ar.p, 0, sizeof(double) * 3 * n, st));
    MD_CUDA(cudaMemsetAsync(a->av.p, 0, sizeof(double) * 3 * n, st));
    MD_CUDA(cudaMemsetAsync(a->scal.p + kS_THETA, 0, 2 * sizeof(double), st));
    const int segments = static_cast<int>((a->steps + a->every - 1) / a->every);
    const unsigned g3 = blocks_for(3ll * a->n, kThreads);
    for (int sg = segments - 1; sg >= 0; --sg) {
        const int k0 = sg * a->every, k1 = std::min(a->steps, k0 + a->every);
        // recompute the segment from its checkpoint
        MD_TRY(async_copy(a->pos.p, a->ck_pos[sg]->p, sizeof(double4) * n, st));
        MD_TRY(async_copy(a->vel.p, a->ck_vel[sg]->p, sizeof(double) * 3 * n, st));
        MD_TRY(adj_build(a, a->ck_ref[sg]->p));
        int gen = 0;
        MD_TRY(keep(a->gen_ref, 0, n));
        MD_TRY(async_copy(a->gen_ref[0]->p, a->ref.p, sizeof(double4) * n, st));
        MD_TRY(adj_forces(a));
        a->seg_gen.assign(k1 - k0 + 1, 0);
        MD_TRY(keep(a->seg_pos, 0, n));
        MD_TRY(keep(a->seg_vel, 0, 3 * n));
        MD_TRY(async_copy(a->seg_pos[0]->p, a->pos.p, sizeof(double4) * n, st));
        MD_TRY(async_copy(a->seg_vel[0]->p, a->vel.p, sizeof(double) * 3 * n, st));
        for (int k = k0 + 1; k <= k1; ++k) {
            bool rebuilt = false;
            MD_TRY(adj_step(a, &rebuilt));
            if (rebuilt) {
                ++gen;
                MD_TRY(keep(a->gen_ref, gen, n));
                MD_TRY(async_copy(a->gen_ref[gen]->p, a->ref.p, sizeof(double4) * n, st));
            }
            const size_t t = k - k0;
            MD_TRY(keep(a->seg_pos, t, n));
            MD_TRY(keep(a->seg_vel, t, 3 * n));
            MD_TRY(async_copy(a->seg_pos[t]->p, a->pos.p, sizeof(double4) * n, st));
            MD_TRY(async_copy(a->seg_vel[t]->p, a->vel.p, sizeof(double) * 3 * n, st));
            a->seg_gen[t] = gen;
        }
        int cur = gen;  // the list currently built
        auto ensure = [&](int want) -> md_status {
            if (want == cur) return MD_OK;
            MD_TRY(adj_build(a, a->gen_ref[want]->p));
            cur = want;
            return MD_OK;
        };
        for (int j = k1; j > k0; --j) {
            const int t = j - k0;
            k_adj_obj_v<<<g3, kThreads, 0, st>>>(a->av.p, a->seg_vel[t]->p, a->mass.p, a->n, aK);
            MD_CHECK_LAUNCH();
            MD_TRY(adj_weights(a));
            MD_TRY(ensure(a->seg_gen[t]));
            MD_TRY(adj_pass(a, a->seg_pos[t]->p, aU, aW, objective));
            k_adj_drift_back<<<g3, kThreads, 0, st>>>(a->av.p, a->ar.p, a->n, a->dt);
            MD_CHECK_LAUNCH();
            MD_TRY(adj_weights(a));
            MD_TRY(ensure(a->seg_gen[t - 1]));
            MD_TRY(adj_pass(a, a->seg_pos[t - 1]->p, 0.0, 0.0, false));
        }
    }
    return MD_OK;
}

}  // namespace

extern "C" {

md_status md_adjoint_create(int device, int64_t n, double box_length, const double* pos4, const double* vel3,
                            const double* mass, double epsilon, double sigma, double cutoff, double skin, double dt,
                            int steps, int checkpoint_every, md_adjoint** out) {
    if (!out || n < 2 || n > kMaxParticles || !pos4 || !vel3 || !(box_length > 0.0) || !(epsilon > 0.0) ||
        !(sigma > 0.0) || !(cutoff > 0.0) || !(skin > 0.0) || !(dt > 0.0) || steps <= 0 || checkpoint_every <= 0)
        return fail(MD_ERR_INVALID, "md_adjoint_create: bad arguments");
    if (2.0 * cutoff > box_length) return fail(MD_ERR_CUTOFF, "Cutoff must be less than half the box length");
    if (2.0 * (cutoff + skin) > box_length)
        return fail(MD_ERR_LIST_RADIUS, "Cutoff + skin must be less than half the box length");
    if (md_device_count() <= device || device < 0) return fail(MD_ERR_NO_DEVICE, "no CUDA device " + std::to_string(device));
    MD_TRY(use_device(device));
    auto* a = new md_adjoint;
    g_launches = &a->launches;
    a->device = device;
    a->n = static_cast<int>(n);
    a->box = Box{box_length, 1.0 / box_length, 0.25 * box_length};
    a->volume = box_length * box_length * box_length;
    a->eps = epsilon;
    a->sigma = sigma;
    a->rc = cutoff;
    a->skin = skin;
    a->dt = dt;
    a->steps = steps;
    a->every = checkpoint_every;
    a->rl2 = (cutoff + skin) * (cutoff + skin);
    a->max_disp2 = 0.25 * skin * skin;  // src/NeighbourList.cpp:7
    a->half_dt = 0.5 * dt;
    adj_constants(a);
    {
        const double rho = static_cast<double>(n) / a->volume;
        const double rl = cutoff + skin;
        const double est = std::min(4.18879020478639 * rl * rl * rl * rho, static_cast<double>(n));
        a->cap = ((static_cast<int>(1.35 * est) + 24) + 7) & ~7;
    }
    md_status st = MD_OK;
    auto chk = [&](cudaError_t e) {
        if (e != cudaSuccess && st == MD_OK) st = fail(MD_ERR_CUDA, cudaGetErrorString(e));
    };
    const size_t N = static_cast<size_t>(n);
    chk(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking));
    for (auto* b : {&a->pos, &a->pos0, &a->ref}) chk(b->reserve(N));
    for (auto* b : {&a->vel, &a->vel0, &a->force, &a->ar, &a->av, &a->wv}) chk(b->reserve(3 * N));
    for (auto* b : {&a->mass, &a->u, &a->w, &a->pe, &a->ps, &a->us, &a->ws, &a->ue, &a->we}) chk(b->reserve(N));
    chk(a->counts.reserve(N));
    chk(a->flags.reserve(2));
    chk(a->blocks.reserve((N + kChunk - 1) / kChunk));
    chk(a->scal.reserve(16));
    chk(cudaMallocHost(reinterpret_cast<void**>(&a->h_flag), sizeof(int)));
    if (st == MD_OK) {
        chk(cudaMemcpyAsync(a->pos0.p, pos4, sizeof(double4) * N, cudaMemcpyHostToDevice, a->stream));
        chk(cudaMemcpyAsync(a->vel0.p, vel3, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, a->stream));
        std::vector<double> m(N, 1.0);
        if (mass) m.assign(mass, mass + N);
        chk(cudaMemcpyAsync(a->mass.p, m.data(), sizeof(double) * N, cudaMemcpyHostToDevice, a->stream));
        chk(cudaFuncSetAttribute(k_adj_blocks2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(4 * kChunk * sizeof(double2))));
        chk(cudaStreamSynchronize(a->stream));
    }
    if (st != MD_OK) {
        g_launches = nullptr;
        delete a;
        return st;
    }
    *out = a;
    return MD_OK;
}

md_status md_adjoint_destroy(md_adjoint* a) {
    if (a) {
        if (g_launches == &a->launches) g_launches = nullptr;
        cudaSetDevice(a->device);
        delete a;
    }
    return MD_OK;
}

md_status md_adjoint_set_parameters(md_adjoint* a, double epsilon, double sigma) {
    if (!a || !(epsilon > 0.0) || !(sigma > 0.0)) return fail(MD_ERR_INVALID, "md_adjoint_set_parameters: bad arguments");
    a->eps = epsilon;
    a->sigma = sigma;
    adj_constants(a);
    a->forwarded = false;
    return MD_OK;
}

md_status md_adjoint_set_state(md_adjoint* a, const double* pos4, const double* vel3) {
    if (!a) return fail(MD_ERR_INVALID, "null adjoint");
    MD_TRY(use_adjoint(a));
    const size_t N = static_cast<size_t>(a->n);
    if (pos4) MD_CUDA(cudaMemcpyAsync(a->pos0.p, pos4, sizeof(double4) * N, cudaMemcpyHostToDevice, a->stream));
    if (vel3) MD_CUDA(cudaMemcpyAsync(a->vel0.p, vel3, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, a->stream));
    MD_CUDA(cudaStreamSynchronize(a->stream));
    a->forwarded = false;
    return MD_OK;
}

md_status md_adjoint_forward(md_adjoint* a, double* mean_pe, double* mean_pressure, double* pe_steps, double* w_steps,
                             double* ke_steps) {
    if (!a) return fail(MD_ERR_INVALID, "null adjoint");
    MD_TRY(use_adjoint(a));
    MD_TRY(adj_forward(a));
    if (mean_pe) *mean_pe = a->meanU;
    if (mean_pressure) *mean_pressure = a->meanP;
    const size_t K = static_cast<size_t>(a->steps);
    if (pe_steps) MD_CUDA(cudaMemcpyAsync(pe_steps, a->U.p + 1, sizeof(double) * K, cudaMemcpyDeviceToHost, a->stream));
    if (w_steps) MD_CUDA(cudaMemcpyAsync(w_steps, a->W.p + 1, sizeof(double) * K, cudaMemcpyDeviceToHost, a->stream));
    if (ke_steps) MD_CUDA(cudaMemcpyAsync(ke_steps, a->KE.p + 1, sizeof(double) * K, cudaMemcpyDeviceToHost, a->stream));
    MD_CUDA(cudaStreamSynchronize(a->stream));
    return MD_OK;
}

md_status md_adjoint_backward(md_adjoint* a, double g_pe, double g_pressure, double* d_epsilon, double* d_sigma,
                              double* d_pos3, double* d_vel3) {
    if (!a) return fail(MD_ERR_INVALID, "null adjoint");
    if (!a->forwarded) return fail(MD_ERR_STATE, "md_adjoint_backward needs md_adjoint_forward first");
    MD_TRY(use_adjoint(a));
    MD_TRY(adj_backward(a, g_pe, g_pressure));
    double theta[2];
    MD_CUDA(cudaMemcpyAsync(theta, a->scal.p + kS_THETA, sizeof(theta), cudaMemcpyDeviceToHost, a->stream));
    const size_t N = static_cast<size_t>(a->n);
    if (d_pos3) MD_CUDA(cudaMemcpyAsync(d_pos3, a->ar.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, a->stream));
    if (d_vel3) MD_CUDA(cudaMemcpyAsync(d_vel3, a->av.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, a->stream));
    MD_CUDA(cudaStreamSynchronize(a->stream));
    if (d_epsilon) *d_epsilon = theta[0];
    if (d_sigma) *d_sigma = theta[1];
    return MD_OK;
}

md_status md_adjoint_info(const md_adjoint* a, int64_t* n, int* steps, int* checkpoint_every, int* rebuilds,
                          uint64_t* launches) {
    if (!a) return fail(MD_ERR_INVALID, "null adjoint");
    if (n) *n = a->n;
    if (steps) *steps = a->steps;
    if (checkpoint_every) *checkpoint_every = a->every;
    if (rebuilds) *rebuilds = a->rebuilds;
    if (launches) *launches = a->launches;
    return MD_OK;
}

}  // extern "C"
