// Host orchestration of batched replicas (md_batch_* in include/md_b200.h). Included at the end of md_abi.cu.
//
// A run is cut into chunks of steps; each chunk is one CUDA graph (captured once per chunk length) whose steps
// need no host decision: rebuilds are chosen per replica on the device (md_batch.cuh). Before a chunk the host
// uploads the chunk's Bussi draws (drawn per replica from std::mt19937_64 like md_bussi_noise, while the
// previous chunk runs) and copies the state to a device snapshot. A neighbour row that outgrew the capacity
// inside a chunk is detected afterwards; the state is restored, the capacity grown and the chunk run again,
// which reproduces the same trajectory.

#include <map>

struct md_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    int R = 0;
    int64_t atoms = 0;
    int slots = 0, tiles = 0, cells = 0, chunks = 0;
    std::vector<BRep> reps_h;
    DevBuf<BRep> reps;
    DevBuf<int> tile_rep, chunk_rep;
    md_batch_options opt{};
    LJ lj{};
    FloatLJ flj{};
    double rl2 = 0.0, max_disp2 = 0.0, bussi_c = 0.0;
    int chunk = 0;        // steps per graph
    int thermo_every = 0; // thermostat period in steps (0: none)
    // particle slots
    DevBuf<double4> pos, pos2, ref_pos;
    DevBuf<double> vel, vel2, force, force2, mass, mass2;
    DevBuf<uint64_t> ids, ids2;
    DevBuf<float4> frames;
    DevBuf<int> cell_of, cell_sorted, half_off;
    DevBuf<uint32_t> bucket, order, rows;
    DevBuf<int2> counts;
    int cap = 0;
    // cells
    DevBuf<int> count, cursor, start;
    // per replica
    DevBuf<int> stale, stale_reps, stale_tiles, work, pairs, item_off, flags;
    DevBuf<unsigned long long> acc, rebuilds, inside;
    DevBuf<double> ke, chunk_sums, noise, rec, tmp_pe, tmp_w;
    DevBuf<double2> scale, item_sums;
    // snapshot at the start of a chunk
    DevBuf<double4> s_pos, s_ref;
    DevBuf<double> s_vel, s_force, s_mass;
    DevBuf<uint64_t> s_ids;
    DevBuf<int> s_cell;
    DevBuf<int2> s_counts;
    DevBuf<uint32_t> s_rows;
    DevBuf<double2> s_scale;
    DevBuf<unsigned long long> s_rebuilds;
    // host side
    std::vector<std::mt19937_64> rng;
    double* h_noise = nullptr;  // pinned: two chunks of draws
    double* h_rec = nullptr;    // pinned: one chunk of records
    int* h_flags = nullptr;     // pinned
    std::map<int, std::pair<cudaGraphExec_t, uint64_t>> graphs;  // chunk length -> (graph, kernels in it)
    struct Variant {
        int apb, tpa;
        bool prefetch;
    };
    std::vector<Variant> variants;
    int variant = 0;
    // tuned on the replicas' starting state (often a lattice); tuned again once after the first chunk of the
    // first run, on a state the dynamics has reached, unless md_batch_set_force_variant pinned one
    bool retuned = false;
    uint64_t launches = 0;
    ~md_batch() {
        for (auto& g : graphs) cudaGraphExecDestroy(g.second.first);
        if (h_noise) cudaFreeHost(h_noise);
        if (h_rec) cudaFreeHost(h_rec);
        if (h_flags) cudaFreeHost(h_flags);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

constexpr int kMaxAttempts = 4;
constexpr int kRecRows = 4;  // per recorded step: potential energy, virial, kinetic energy, inside-cutoff pairs

// Steps per chunk graph: chunk_steps (100 by default) rounded up to a multiple of the sampling and thermostat
// periods, so every chunk starts on a multiple of both
int b_chunk_len(const md_batch_options& o, int thermo_every) {
    auto gcd = [](int64_t x, int64_t y) {
        while (y) {
            const int64_t t = x % y;
            x = y;
            y = t;
        }
        return x;
    };
    int64_t period = 1;
    for (int64_t p : {static_cast<int64_t>(o.energy_every), static_cast<int64_t>(thermo_every)})
        if (p > 0) period = period / gcd(period, p) * p;
    int64_t want = o.chunk_steps > 0 ? o.chunk_steps : 100;
    want = (want + period - 1) / period * period;
    return static_cast<int>(std::min<int64_t>(want, 1 << 20));
}

// The buffers sized by the chunk length: Bussi draws (device, and two chunks' worth pinned on the host) and the
// records of one chunk (device and pinned host)
md_status b_chunk_buffers(md_batch* b) {
    const size_t R = static_cast<size_t>(b->R), C = static_cast<size_t>(b->chunk);
    const int every = b->opt.energy_every;
    const size_t samples = every > 0 ? C / every : 0;
    MD_CUDA(b->noise.reserve(2 * C * R));
    MD_CUDA(b->rec.reserve(std::max<size_t>(1, kRecRows * samples * R)));
    if (b->h_noise) cudaFreeHost(b->h_noise);
    if (b->h_rec) cudaFreeHost(b->h_rec);
    b->h_noise = b->h_rec = nullptr;
    MD_CUDA(cudaMallocHost(reinterpret_cast<void**>(&b->h_noise), sizeof(double) * 4 * C * R));
    MD_CUDA(cudaMallocHost(reinterpret_cast<void**>(&b->h_rec), sizeof(double) * std::max<size_t>(1, kRecRows * samples * R)));
    return MD_OK;
}

md_status use_batch(md_batch* b) {
    g_launches = &b->launches;
    MD_CUDA(cudaSetDevice(b->device));
    return MD_OK;
}

md_status bsync(md_batch* b) {
    MD_CUDA(cudaStreamSynchronize(b->stream));
    MD_CUDA(cudaGetLastError());
    return MD_OK;
}

unsigned rebuild_grid(const md_batch* b) { return static_cast<unsigned>(std::min(b->tiles, 148 * 8)); }
unsigned replica_grid(const md_batch* b) { return static_cast<unsigned>(std::min(b->R, 148 * 4)); }
unsigned per_replica(const md_batch* b, int threads) { return blocks_for(b->R, threads); }

bool float_mode(const md_batch* b) { return b->opt.precision != MD_PREC_FP64; }

// The list rebuild of every replica flagged stale (all of them when the flags were set by the host)
md_status b_rebuild_async(md_batch* b) {
    cudaStream_t st = b->stream;
    k_b_stale_lists<<<1, kListThreads, 0, st>>>(b->reps.p, b->R, b->stale.p, b->stale_reps.p, b->stale_tiles.p,
                                                 b->work.p, b->rebuilds.p);
    MD_CHECK_LAUNCH();
    const unsigned gt = rebuild_grid(b), gr = replica_grid(b);
    k_b_cell_assign<<<gt, kTile, 0, st>>>(b->reps.p, b->tile_rep.p, b->stale_tiles.p, b->work.p, b->pos.p, b->cell_of.p,
                                          b->count.p);
    MD_CHECK_LAUNCH();
    k_b_cell_scan<<<gr, kRepScanThreads, 0, st>>>(b->reps.p, b->stale_reps.p, b->work.p, b->count.p, b->start.p);
    MD_CHECK_LAUNCH();
    k_b_cell_scatter<<<gt, kTile, 0, st>>>(b->reps.p, b->tile_rep.p, b->stale_tiles.p, b->work.p, b->cell_of.p,
                                           b->start.p, b->cursor.p, b->bucket.p);
    MD_CHECK_LAUNCH();
    k_b_cell_rank<<<gt, kTile, 0, st>>>(b->reps.p, b->tile_rep.p, b->stale_tiles.p, b->work.p, b->cell_of.p,
                                        b->start.p, b->cursor.p, b->bucket.p, b->order.p);
    MD_CHECK_LAUNCH();
    k_b_permute<<<gt, kTile, 0, st>>>(b->reps.p, b->tile_rep.p, b->stale_tiles.p, b->work.p, b->order.p, b->cell_of.p,
                                      b->pos.p, b->vel.p, b->force.p, b->mass.p, b->ids.p, b->pos2.p, b->vel2.p,
                                      b->force2.p, b->mass2.p, b->ids2.p, b->cell_sorted.p);
    MD_CHECK_LAUNCH();
    k_b_commit<<<gt, kTile, 0, st>>>(b->reps.p, b->tile_rep.p, b->stale_tiles.p, b->work.p, b->pos2.p, b->vel2.p,
                                     b->force2.p, b->mass2.p, b->ids2.p, b->cell_sorted.p, b->pos.p, b->vel.p,
                                     b->force.p, b->mass.p, b->ids.p, b->ref_pos.p, b->frames.p);
    MD_CHECK_LAUNCH();
    const double rl2 = b->rl2;
    const double margin = 1e-5 * rl2 + 1e-4;  // bound on the float r^2 error of fresh frames (as the tile build)
    const BBuild bp{rl2, static_cast<float>(rl2 - margin), static_cast<float>(rl2 + margin), b->cap,
                    static_cast<uint32_t>(b->slots) | (kSentinelCode << kCodeShift)};
    k_b_nlist_build<<<gt, kTile, 0, st>>>(b->reps.p, b->tile_rep.p, b->stale_tiles.p, b->work.p, b->pos.p, b->frames.p,
                                          b->cell_sorted.p, b->start.p, bp, b->rows.p, b->counts.p, b->flags.p);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

template <bool kFixed, bool kEnergy>
md_status b_float_forces(md_batch* b, const md_batch::Variant& v, bool kick) {
    const unsigned grid = static_cast<unsigned>(b->tiles) * (kTile / v.apb);
    const int threads = v.apb * v.tpa;
    double* kv = kick ? b->vel.p : nullptr;
    const double half_dt = 0.5 * b->opt.dt;
#define MD_B_FORCE(T, P)                                                                                              \
    k_b_force_fp32<kFixed, kEnergy, T, P><<<grid, threads, 0, b->stream>>>(                                           \
        b->reps.p, b->tile_rep.p, v.apb, b->frames.p, b->pos.p, b->flj, b->rows.p, b->cap, b->counts.p, b->force.p, \
        b->acc.p, kv, b->mass.p, half_dt)
    if (v.tpa == 1) {
        if (v.prefetch) MD_B_FORCE(1, true);
        else MD_B_FORCE(1, false);
    } else if constexpr (kFixed) {
        if (v.tpa == 2) MD_B_FORCE(2, false);
        else MD_B_FORCE(4, false);
    } else {
        return fail(MD_ERR_INVALID, "float accumulation runs one thread per particle");
    }
#undef MD_B_FORCE
    MD_CHECK_LAUNCH();
    return MD_OK;
}

// List forces of every replica with the given kernel variant; with `kick` the closing half kick (and, in float
// modes, the fused fixed-point kinetic energy); with `energy` the float energy/virial sums
md_status b_forces(md_batch* b, int variant, bool kick, bool energy) {
    if (!float_mode(b)) {
        k_b_force_fp64<<<b->tiles, kTile, 0, b->stream>>>(b->reps.p, b->tile_rep.p, b->pos.p, b->lj, b->rows.p, b->cap,
                                                          b->counts.p, b->force.p, b->acc.p, kick ? b->vel.p : nullptr,
                                                          b->mass.p, 0.5 * b->opt.dt);
        MD_CHECK_LAUNCH();
        return MD_OK;
    }
    const md_batch::Variant& v = b->variants[variant];
    const bool fixed = b->opt.precision == MD_PREC_FP32FX;
    if (fixed) return energy ? b_float_forces<true, true>(b, v, kick) : b_float_forces<true, false>(b, v, kick);
    return energy ? b_float_forces<false, true>(b, v, kick) : b_float_forces<false, false>(b, v, kick);
}

// FP64 kinetic energies in the reference's blocked order into `out` (with the pending scale applied if asked)
md_status b_kinetic_fp64(md_batch* b, bool scaled, double* out) {
    const size_t smem = kEnergyWarps * kChunk * sizeof(double);
    k_b_kinetic_blocks<<<blocks_for(b->chunks, kEnergyWarps), kEnergyWarps * 32, smem, b->stream>>>(
        b->reps.p, b->chunk_rep.p, b->chunks, b->vel.p, b->mass.p, scaled ? b->scale.p : nullptr, b->chunk_sums.p);
    MD_CHECK_LAUNCH();
    k_b_sum_chunks<<<blocks_for(static_cast<long long>(b->R) * 32, kThreads), kThreads, 0, b->stream>>>(
        b->reps.p, b->R, b->chunk_sums.p, out);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

// FP64 energy and virial of every replica in the reference's pair order into pe_out / w_out
md_status b_energy_fp64(md_batch* b, double* pe_out, double* w_out) {
    k_b_half_offsets<<<replica_grid(b), kRepScanThreads, 0, b->stream>>>(b->reps.p, b->R, b->counts.p, b->half_off.p,
                                                                      b->pairs.p);
    MD_CHECK_LAUNCH();
    k_b_pair_items<<<1, kRepScanThreads, 0, b->stream>>>(b->R, b->pairs.p, b->item_off.p);
    MD_CHECK_LAUNCH();
    const size_t smem = kEnergyWarps * kChunk * sizeof(double2);
    k_b_energy_blocks<<<148 * 4, kEnergyWarps * 32, smem, b->stream>>>(b->reps.p, b->R, b->item_off.p, b->pairs.p,
                                                                       b->half_off.p, b->pos.p, b->lj, b->rows.p,
                                                                       b->cap, b->item_sums.p);
    MD_CHECK_LAUNCH();
    k_b_sum_items<<<blocks_for(static_cast<long long>(b->R) * 32, kThreads), kThreads, 0, b->stream>>>(
        b->R, b->item_off.p, b->item_sums.p, pe_out, w_out);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

// Energy, virial and inside count from the last force evaluation plus the kinetic energy after any pending
// scale, into the given device arrays (R each)
md_status b_observables(md_batch* b, double* pe_out, double* w_out, double* ke_out) {
    if (float_mode(b)) {
        // the float energy sums were accumulated by the force launch; the kinetic energy is recomputed
        k_b_kinetic_fixed<<<b->tiles, kTile, 0, b->stream>>>(b->reps.p, b->tile_rep.p, b->vel.p, b->mass.p,
                                                             b->scale.p, b->acc.p);
        MD_CHECK_LAUNCH();
        k_b_finish_float<<<per_replica(b, kThreads), kThreads, 0, b->stream>>>(b->R, b->acc.p, true, ke_out, pe_out,
                                                                               w_out, b->inside.p);
        MD_CHECK_LAUNCH();
        return MD_OK;
    }
    k_b_finish_fp64<<<per_replica(b, kThreads), kThreads, 0, b->stream>>>(b->R, b->acc.p, b->inside.p);
    MD_CHECK_LAUNCH();
    MD_TRY(b_energy_fp64(b, pe_out, w_out));
    return b_kinetic_fp64(b, true, ke_out);
}

// One step of every replica (src/Integrator.cpp:18-30, then the thermostat); `k` is the step's index in its
// chunk, `step` its number in the run (1-based), `rec` the sample's records or null.
md_status b_enqueue_step(md_batch* b, int k, int64_t step, double* rec) {
    cudaStream_t st = b->stream;
    const bool fl = float_mode(b);
    const double dt = b->opt.dt;
#define MD_B_DRIFT(F)                                                                                                \
    k_b_kick_drift<F><<<b->tiles, kTile, 0, st>>>(b->reps.p, b->tile_rep.p, b->pos.p, b->vel.p, b->force.p,           \
                                                  b->mass.p, 0.5 * dt, dt, b->ref_pos.p, b->max_disp2, b->stale.p,     \
                                                  b->scale.p, b->cell_sorted.p, b->frames.p)
    if (fl) MD_B_DRIFT(true);
    else MD_B_DRIFT(false);
#undef MD_B_DRIFT
    MD_CHECK_LAUNCH();
    // a thermostat applied in the previous step has been consumed by the drift. Chunks start on multiples of
    // the period, so the step before step 1 of a chunk may have been a thermostat step (clearing is harmless
    // when nothing is pending).
    const bool thermo = b->thermo_every > 0 && step % b->thermo_every == 0;
    const bool thermo_prev = b->thermo_every > 0 && (step - 1) % b->thermo_every == 0;
    if (thermo_prev && !thermo) {
        k_b_clear_scale<<<per_replica(b, kThreads), kThreads, 0, st>>>(b->R, b->scale.p);
        MD_CHECK_LAUNCH();
    }
    MD_TRY(b_rebuild_async(b));
    const bool sample = rec != nullptr;
    MD_TRY(b_forces(b, b->variant, true, sample && fl));
    const int R = b->R;
    if (fl) {
        k_b_finish_float<<<per_replica(b, kThreads), kThreads, 0, st>>>(R, b->acc.p, true, b->ke.p,
                                                                        sample ? rec : nullptr,
                                                                        sample ? rec + R : nullptr, b->inside.p);
        MD_CHECK_LAUNCH();
    } else {
        k_b_finish_fp64<<<per_replica(b, kThreads), kThreads, 0, st>>>(R, b->acc.p, b->inside.p);
        MD_CHECK_LAUNCH();
        if (thermo) MD_TRY(b_kinetic_fp64(b, false, b->ke.p));
        if (sample) MD_TRY(b_energy_fp64(b, rec, rec + R));
    }
    if (sample) {
        k_b_record_inside<<<per_replica(b, kThreads), kThreads, 0, st>>>(R, b->inside.p, rec + 3 * R);
        MD_CHECK_LAUNCH();
    }
    if (thermo) {
        const double* r1 = b->noise.p + static_cast<size_t>(k) * R;
        const double* chi2 = b->noise.p + static_cast<size_t>(b->chunk + k) * R;
        k_b_thermostat<<<per_replica(b, kThreads), kThreads, 0, st>>>(b->reps.p, R, b->opt.thermostat, b->ke.p,
                                                                      b->bussi_c, r1, chi2, b->scale.p);
        MD_CHECK_LAUNCH();
    }
    if (sample) {
        if (fl) {
            k_b_kinetic_fixed<<<b->tiles, kTile, 0, st>>>(b->reps.p, b->tile_rep.p, b->vel.p, b->mass.p, b->scale.p,
                                                          b->acc.p);
            MD_CHECK_LAUNCH();
            k_b_finish_float<<<per_replica(b, kThreads), kThreads, 0, st>>>(R, b->acc.p, true, rec + 2 * R, nullptr,
                                                                            nullptr, nullptr);
            MD_CHECK_LAUNCH();
        } else {
            MD_TRY(b_kinetic_fp64(b, true, rec + 2 * R));
        }
    }
    return MD_OK;
}

// The graph of `len` steps (recorded energies at every energy_every-th step into rec[(s * kRecRows + q) * R + r])
md_status b_graph(md_batch* b, int len, cudaGraphExec_t* out, uint64_t* kernels) {
    auto it = b->graphs.find(len);
    if (it != b->graphs.end()) {
        *out = it->second.first;
        *kernels = it->second.second;
        return MD_OK;
    }
    uint64_t count = 0;
    uint64_t* saved = g_launches;
    g_launches = &count;
    cudaGraph_t graph = nullptr;
    MD_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    md_status st = MD_OK;
    const int every = b->opt.energy_every;
    for (int k = 0; k < len && st == MD_OK; ++k) {
        const int64_t step = k + 1;  // chunks start at multiples of the thermostat and sampling periods
        double* rec = every > 0 && step % every == 0 ? b->rec.p + static_cast<size_t>(step / every - 1) * kRecRows * b->R
                                                     : nullptr;
        st = b_enqueue_step(b, k, step, rec);
    }
    const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    g_launches = saved;
    if (st != MD_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return fail(MD_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return fail(MD_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
    b->graphs[len] = {exec, count};
    *out = exec;
    *kernels = count;
    return MD_OK;
}

void b_drop_graphs(md_batch* b) {
    for (auto& g : b->graphs) cudaGraphExecDestroy(g.second.first);
    b->graphs.clear();
}

md_status b_copy(void* dst, const void* src, size_t bytes, md_batch* b) {
    MD_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, b->stream));
    return MD_OK;
}

// Everything a chunk changes that the next steps read: particle arrays, list, pending scales, rebuild counts
md_status b_snapshot(md_batch* b, bool restore) {
    const size_t S = static_cast<size_t>(b->slots);
    auto pair = [&](void* live, void* saved, size_t bytes) {
        return restore ? b_copy(live, saved, bytes, b) : b_copy(saved, live, bytes, b);
    };
    MD_TRY(pair(b->pos.p, b->s_pos.p, sizeof(double4) * S));
    MD_TRY(pair(b->ref_pos.p, b->s_ref.p, sizeof(double4) * S));
    MD_TRY(pair(b->vel.p, b->s_vel.p, sizeof(double) * 3 * S));
    MD_TRY(pair(b->force.p, b->s_force.p, sizeof(double) * 3 * S));
    MD_TRY(pair(b->mass.p, b->s_mass.p, sizeof(double) * S));
    MD_TRY(pair(b->ids.p, b->s_ids.p, sizeof(uint64_t) * S));
    MD_TRY(pair(b->cell_sorted.p, b->s_cell.p, sizeof(int) * S));
    MD_TRY(pair(b->counts.p, b->s_counts.p, sizeof(int2) * S));
    MD_TRY(pair(b->rows.p, b->s_rows.p, sizeof(uint32_t) * row_buffer_entries(b->slots, b->cap)));
    MD_TRY(pair(b->scale.p, b->s_scale.p, sizeof(double2) * b->R));
    MD_TRY(pair(b->rebuilds.p, b->s_rebuilds.p, sizeof(unsigned long long) * b->R));
    return MD_OK;
}

// 1024-pair blocks of the FP64 energy sums: a replica has at most n cap own pairs
md_status b_alloc_items(md_batch* b) {
    const int64_t items = static_cast<int64_t>(b->slots) * b->cap / kChunk + b->R + 1;
    if (items > INT32_MAX) return fail(MD_ERR_INVALID, "too many neighbour pairs");
    MD_CUDA(b->item_sums.reserve(static_cast<size_t>(items)));
    return MD_OK;
}

md_status b_alloc_rows(md_batch* b) {
    const size_t e = row_buffer_entries(b->slots, b->cap);
    MD_CUDA(b->rows.reserve(e));
    MD_CUDA(b->s_rows.reserve(e));
    return b_alloc_items(b);
}

// Restores the snapshot with rows laid out for a capacity grown to fit `need` entries
md_status b_grow_and_restore(md_batch* b, int need) {
    const int cap0 = b->cap;
    const int cap1 = ((need + need / 4 + 16) + 7) & ~7;
    // the restored counts are the snapshot's: relayout the snapshot rows into a new live buffer
    MD_TRY(b_copy(b->counts.p, b->s_counts.p, sizeof(int2) * b->slots, b));
    DevBuf<uint32_t> fresh;
    MD_CUDA(fresh.reserve(row_buffer_entries(b->slots, cap1)));
    k_b_relayout_rows<<<blocks_for(b->slots, kThreads), kThreads, 0, b->stream>>>(b->slots, b->counts.p, b->s_rows.p,
                                                                                  cap0, fresh.p, cap1);
    MD_CHECK_LAUNCH();
    MD_TRY(bsync(b));
    std::swap(b->rows.p, fresh.p);
    std::swap(b->rows.count, fresh.count);
    b->cap = cap1;
    b->s_rows.release();
    MD_CUDA(b->s_rows.reserve(row_buffer_entries(b->slots, cap1)));
    MD_TRY(b_alloc_items(b));
    // the rows are now current; restore the rest and re-take the snapshot with the new layout
    const size_t S = static_cast<size_t>(b->slots);
    MD_TRY(b_copy(b->pos.p, b->s_pos.p, sizeof(double4) * S, b));
    MD_TRY(b_copy(b->ref_pos.p, b->s_ref.p, sizeof(double4) * S, b));
    MD_TRY(b_copy(b->vel.p, b->s_vel.p, sizeof(double) * 3 * S, b));
    MD_TRY(b_copy(b->force.p, b->s_force.p, sizeof(double) * 3 * S, b));
    MD_TRY(b_copy(b->mass.p, b->s_mass.p, sizeof(double) * S, b));
    MD_TRY(b_copy(b->ids.p, b->s_ids.p, sizeof(uint64_t) * S, b));
    MD_TRY(b_copy(b->cell_sorted.p, b->s_cell.p, sizeof(int) * S, b));
    MD_TRY(b_copy(b->scale.p, b->s_scale.p, sizeof(double2) * b->R, b));
    MD_TRY(b_copy(b->rebuilds.p, b->s_rebuilds.p, sizeof(unsigned long long) * b->R, b));
    MD_TRY(b_copy(b->s_rows.p, b->rows.p, sizeof(uint32_t) * row_buffer_entries(b->slots, cap1), b));
    MD_CUDA(cudaMemsetAsync(b->stale.p, 0, sizeof(int) * b->R, b->stream));
    b_drop_graphs(b);
    return bsync(b);
}

// The chunk's thermostat draws for every replica (md_bussi_noise's sequence, continued per replica)
void b_draw(md_batch* b, int len, double* host) {
    if (b->opt.thermostat != 2) return;
    const int R = b->R;
    for (int r = 0; r < R; ++r) {
        const double dof = b->reps_h[r].dof;
        for (int k = 0; k < len; ++k) {
            std::normal_distribution<double> gaussian(0.0, 1.0);
            std::gamma_distribution<double> gamma(0.5 * (dof - 1.0), 2.0);
            host[static_cast<size_t>(k) * R + r] = gaussian(b->rng[r]);
            host[static_cast<size_t>(b->chunk + k) * R + r] = gamma(b->rng[r]);
        }
    }
}

// Times every force variant (no kick, no energy) and keeps the fastest; all variants give the same bits
md_status b_autotune(md_batch* b) {
    if (b->variants.size() <= 1) {
        b->variant = 0;
        return MD_OK;
    }
    cudaEvent_t e0, e1;
    MD_CUDA(cudaEventCreate(&e0));
    MD_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int pick = 0;
    md_status st = MD_OK;
    for (size_t v = 0; v < b->variants.size() && st == MD_OK; ++v) {
        st = b_forces(b, static_cast<int>(v), false, false);  // warm-up
        if (st != MD_OK) break;
        cudaEventRecord(e0, b->stream);
        for (int rep = 0; rep < 3 && st == MD_OK; ++rep) st = b_forces(b, static_cast<int>(v), false, false);
        cudaEventRecord(e1, b->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = fail(MD_ERR_CUDA, "autotune timing failed");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            pick = static_cast<int>(v);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MD_TRY(st);
    b->variant = pick;
    return MD_OK;
}

// Clears the float sums left by a force launch that did not finish them
md_status b_clear_acc(md_batch* b) {
    MD_CUDA(cudaMemsetAsync(b->acc.p, 0, sizeof(unsigned long long) * 4 * b->R, b->stream));
    return MD_OK;
}

// Host-driven list build of every replica (creation): all flagged stale, rebuilt, grown until the rows fit
md_status b_initial_build(md_batch* b) {
    for (int attempt = 0; attempt < kMaxAttempts; ++attempt) {
        MD_TRY(b_alloc_rows(b));
        std::vector<int> ones(b->R, 1);
        MD_CUDA(cudaMemcpyAsync(b->stale.p, ones.data(), sizeof(int) * b->R, cudaMemcpyHostToDevice, b->stream));
        MD_CUDA(cudaMemsetAsync(b->flags.p, 0, sizeof(int), b->stream));
        MD_TRY(b_rebuild_async(b));
        MD_CUDA(cudaMemcpyAsync(b->h_flags, b->flags.p, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
        MD_TRY(bsync(b));
        if (b->h_flags[0] <= b->cap) {
            // a repeated build sorted an already sorted state (identity order); it counts once
            std::vector<unsigned long long> one(b->R, 1);
            MD_CUDA(cudaMemcpyAsync(b->rebuilds.p, one.data(), sizeof(unsigned long long) * b->R, cudaMemcpyHostToDevice,
                                    b->stream));
            return bsync(b);
        }
        const int need = b->h_flags[0];
        b->cap = ((need + need / 4 + 16) + 7) & ~7;
        b->rows.release();
        b->s_rows.release();
    }
    return fail(MD_ERR_CAPACITY, "neighbour row capacity could not be met");
}

}  // namespace

extern "C" {

md_status md_batch_create(int device, int replicas, const int64_t* n_atoms, const double* box_length,
                          const double* temperature, const uint64_t* seeds, const double* pos4, const double* vel3,
                          const double* mass, const md_batch_options* opts, md_batch** out) {
    if (!out || replicas <= 0 || !n_atoms || !box_length || !pos4 || !opts)
        return fail(MD_ERR_INVALID, "md_batch_create: bad arguments");
    const md_batch_options& o = *opts;
    if (!(o.epsilon > 0.0) || !(o.sigma > 0.0) || !(o.cutoff > 0.0) || !(o.skin > 0.0) || !(o.dt > 0.0) ||
        o.precision < MD_PREC_FP64 || o.precision > MD_PREC_FP32 || o.thermostat < 0 || o.thermostat > 2 ||
        (o.thermostat == 1 && o.rescale_every <= 0) || (o.thermostat == 2 && (!(o.bussi_tau > 0.0) || !seeds)) ||
        (o.thermostat != 0 && !temperature) || o.energy_every < 0 || o.chunk_steps < 0 || o.initial_capacity < 0)
        return fail(MD_ERR_INVALID, "md_batch_create: bad options");
    const double rl = o.cutoff + o.skin;
    int64_t slots = 0, atoms = 0;
    for (int r = 0; r < replicas; ++r) {
        const int64_t n = n_atoms[r];
        const double L = box_length[r];
        if (n < 2 || !(L > 0.0)) return fail(MD_ERR_INVALID, "replica " + std::to_string(r) + ": bad size or box");
        if (2.0 * o.cutoff > L) return fail(MD_ERR_CUTOFF, "replica " + std::to_string(r) + ": cut-off must be at most half the box length");
        if (2.0 * rl > L) return fail(MD_ERR_LIST_RADIUS, "replica " + std::to_string(r) + ": cutoff + skin must be less than half the box length");
        slots += (n + kTile - 1) / kTile * kTile;
        atoms += n;
    }
    if (slots >= kMaxParticles) return fail(MD_ERR_INVALID, "md_batch_create: too many particles");
    if (md_device_count() <= device || device < 0) return fail(MD_ERR_NO_DEVICE, "no CUDA device " + std::to_string(device));
    MD_TRY(use_device(device));
    auto* b = new md_batch;
    b->device = device;
    g_launches = &b->launches;
    b->R = replicas;
    b->opt = o;
    b->atoms = atoms;
    b->slots = static_cast<int>(slots);
    b->tiles = static_cast<int>(slots / kTile);
    // constants as LennardJonesForceField computes them (src/Forcefield.cpp:8-15)
    {
        b->lj = lj_constants(o.epsilon, o.sigma, o.cutoff);
        md_forcefield tmp;
        tmp.lj = b->lj;
        b->flj = float_lj(&tmp);
    }
    b->rl2 = rl * rl;
    b->max_disp2 = 0.25 * o.skin * o.skin;  // src/NeighbourList.cpp:7
    b->bussi_c = o.thermostat == 2 ? std::exp(-o.dt / o.bussi_tau) : 0.0;  // src/Thermostat.cpp:46
    b->thermo_every = o.thermostat == 2 ? 1 : (o.thermostat == 1 ? o.rescale_every : 0);
    b->chunk = b_chunk_len(o, b->thermo_every);
    // layout
    b->reps_h.resize(replicas);
    std::vector<int> tile_rep(b->tiles), chunk_rep;
    int off = 0, cell_off = 0, chunk_off = 0;
    for (int r = 0; r < replicas; ++r) {
        BRep& d = b->reps_h[r];
        const int n = static_cast<int>(n_atoms[r]);
        const double L = box_length[r];
        d.box = Box{L, 1.0 / L, 0.25 * L};
        d.ncps = std::max(1, static_cast<int>(L / rl));  // src/CellList.cpp:14
        d.inv_cell = d.ncps / L;                          // src/CellList.cpp:18
        d.cell = L / d.ncps;
        d.dof = 3.0 * static_cast<double>(n) - 3.0;
        d.temperature = temperature ? temperature[r] : 0.0;
        d.off = off;
        d.n = n;
        d.np = (n + kTile - 1) / kTile * kTile;
        d.ncells = d.ncps * d.ncps * d.ncps;
        d.cell_off = cell_off;
        d.use_cells = d.ncps >= 3 ? 1 : 0;  // src/NeighbourList.cpp:69
        d.tile_off = off / kTile;
        d.chunk_off = chunk_off;
        for (int t = 0; t < d.np / kTile; ++t) tile_rep[d.tile_off + t] = r;
        const int nch = (n + kChunk - 1) / kChunk;
        for (int c = 0; c < nch; ++c) chunk_rep.push_back(r);
        off += d.np;
        cell_off += d.ncells;
        chunk_off += nch;
    }
    b->cells = cell_off;
    b->chunks = chunk_off;
    // initial row capacity: the full r_l sphere at the densest replica with a margin (or the caller's)
    if (o.initial_capacity > 0) {
        b->cap = (o.initial_capacity + 7) & ~7;
    } else {
        double rho_max = 0.0;
        for (const BRep& d : b->reps_h) rho_max = std::max(rho_max, d.n / (d.box.L * d.box.L * d.box.L));
        const double est = 4.18879020478639 * rl * rl * rl * rho_max;
        b->cap = ((static_cast<int>(1.35 * est) + 24) + 7) & ~7;
    }
    md_status st = MD_OK;
    auto chk = [&](cudaError_t e) {
        if (e != cudaSuccess && st == MD_OK) st = fail(MD_ERR_CUDA, cudaGetErrorString(e));
    };
    const size_t S = slots, R = replicas;
    chk(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    chk(b->reps.reserve(R));
    chk(b->tile_rep.reserve(b->tiles));
    chk(b->chunk_rep.reserve(b->chunks));
    for (auto* buf : {&b->pos, &b->pos2, &b->ref_pos, &b->s_pos, &b->s_ref}) chk(buf->reserve(S));
    for (auto* buf : {&b->vel, &b->vel2, &b->force, &b->force2, &b->s_vel, &b->s_force}) chk(buf->reserve(3 * S));
    for (auto* buf : {&b->mass, &b->mass2, &b->s_mass}) chk(buf->reserve(S));
    for (auto* buf : {&b->ids, &b->ids2, &b->s_ids}) chk(buf->reserve(S));
    chk(b->frames.reserve(S + 1));
    for (auto* buf : {&b->cell_of, &b->cell_sorted, &b->half_off, &b->s_cell}) chk(buf->reserve(S));
    chk(b->bucket.reserve(S));
    chk(b->order.reserve(S));
    chk(b->counts.reserve(S));
    chk(b->s_counts.reserve(S));
    chk(b->count.reserve(b->cells));
    chk(b->cursor.reserve(b->cells));
    chk(b->start.reserve(static_cast<size_t>(b->cells) + R));
    for (auto* buf : {&b->stale, &b->stale_reps, &b->pairs}) chk(buf->reserve(R));
    chk(b->stale_tiles.reserve(b->tiles));
    chk(b->work.reserve(2));
    chk(b->item_off.reserve(R + 1));
    chk(b->flags.reserve(1));
    chk(b->acc.reserve(4 * R));
    for (auto* buf : {&b->rebuilds, &b->inside, &b->s_rebuilds}) chk(buf->reserve(R));
    for (auto* buf : {&b->ke, &b->tmp_pe, &b->tmp_w}) chk(buf->reserve(R));
    chk(b->chunk_sums.reserve(b->chunks));
    if (st == MD_OK) st = b_chunk_buffers(b);
    chk(b->scale.reserve(R));
    chk(b->s_scale.reserve(R));
    chk(cudaMallocHost(reinterpret_cast<void**>(&b->h_flags), sizeof(int) * 4));
    if (st == MD_OK) {
        chk(cudaMemcpyAsync(b->reps.p, b->reps_h.data(), sizeof(BRep) * R, cudaMemcpyHostToDevice, b->stream));
        chk(cudaMemcpyAsync(b->tile_rep.p, tile_rep.data(), sizeof(int) * b->tiles, cudaMemcpyHostToDevice, b->stream));
        chk(cudaMemcpyAsync(b->chunk_rep.p, chunk_rep.data(), sizeof(int) * b->chunks, cudaMemcpyHostToDevice, b->stream));
        // particles: the reference layouts per replica into slots; padding slots stay zero with mass 1
        std::vector<double4> hp(S, make_double4(0, 0, 0, 0));
        std::vector<double> hv(3 * S, 0.0), hm(S, 1.0);
        std::vector<uint64_t> hid(S, 0);
        int64_t base = 0;
        for (int r = 0; r < replicas; ++r) {
            const BRep& d = b->reps_h[r];
            for (int i = 0; i < d.n; ++i) {
                const int64_t g = base + i;
                hp[d.off + i] = make_double4(pos4[4 * g], pos4[4 * g + 1], pos4[4 * g + 2], pos4[4 * g + 3]);
                if (mass) hm[d.off + i] = mass[g];
                hid[d.off + i] = static_cast<uint64_t>(i);
                if (vel3)
                    for (int k = 0; k < 3; ++k) hv[3 * static_cast<size_t>(d.off) + static_cast<size_t>(k) * d.np + i] = vel3[3 * base + static_cast<int64_t>(k) * d.n + i];
            }
            base += d.n;
        }
        chk(cudaMemcpyAsync(b->pos.p, hp.data(), sizeof(double4) * S, cudaMemcpyHostToDevice, b->stream));
        chk(cudaMemcpyAsync(b->vel.p, hv.data(), sizeof(double) * 3 * S, cudaMemcpyHostToDevice, b->stream));
        chk(cudaMemcpyAsync(b->mass.p, hm.data(), sizeof(double) * S, cudaMemcpyHostToDevice, b->stream));
        chk(cudaMemcpyAsync(b->ids.p, hid.data(), sizeof(uint64_t) * S, cudaMemcpyHostToDevice, b->stream));
        chk(cudaMemsetAsync(b->force.p, 0, sizeof(double) * 3 * S, b->stream));
        chk(cudaMemsetAsync(b->counts.p, 0, sizeof(int2) * S, b->stream));
        chk(cudaMemsetAsync(b->cell_sorted.p, 0, sizeof(int) * S, b->stream));
        chk(cudaMemsetAsync(b->count.p, 0, sizeof(int) * b->cells, b->stream));
        chk(cudaMemsetAsync(b->cursor.p, 0, sizeof(int) * b->cells, b->stream));
        chk(cudaMemsetAsync(b->acc.p, 0, sizeof(unsigned long long) * 4 * R, b->stream));
        chk(cudaMemsetAsync(b->rebuilds.p, 0, sizeof(unsigned long long) * R, b->stream));
        std::vector<double2> noscale(R, make_double2(1.0, 0.0));
        chk(cudaMemcpyAsync(b->scale.p, noscale.data(), sizeof(double2) * R, cudaMemcpyHostToDevice, b->stream));
        const float4 sentinel = make_float4(kSentinelCoord, kSentinelCoord, kSentinelCoord, 0.0f);
        chk(cudaMemcpyAsync(b->frames.p + S, &sentinel, sizeof(float4), cudaMemcpyHostToDevice, b->stream));
        chk(cudaStreamSynchronize(b->stream));
        chk(cudaFuncSetAttribute(k_b_energy_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kEnergyWarps * kChunk * sizeof(double2))));
    }
    if (st == MD_OK && o.thermostat == 2) {
        b->rng.reserve(replicas);
        for (int r = 0; r < replicas; ++r) b->rng.emplace_back(seeds[r]);
    }
    // force kernel variants: (particles per block, threads per particle)
    if (o.precision == MD_PREC_FP32FX)
        b->variants = {{128, 1, false}, {64, 1, false}, {32, 1, false}, {64, 2, false}, {128, 2, false},
                       {32, 4, false}, {64, 4, false}, {128, 1, true}, {64, 1, true}};
    else if (o.precision == MD_PREC_FP32)
        b->variants = {{128, 1, false}, {64, 1, false}, {32, 1, false}, {128, 1, true}, {64, 1, true}};
    else
        b->variants = {{128, 1, false}};
    if (st == MD_OK) st = b_initial_build(b);
    if (st == MD_OK) st = b_autotune(b);
    if (st == MD_OK) st = b_clear_acc(b);
    // the starting forces from the list (no kick), their sums cleared
    if (st == MD_OK) st = b_forces(b, b->variant, false, false);
    if (st == MD_OK) st = b_clear_acc(b);
    if (st == MD_OK) st = bsync(b);
    if (st != MD_OK) {
        g_launches = nullptr;
        delete b;
        return st;
    }
    *out = b;
    return MD_OK;
}

md_status md_batch_destroy(md_batch* b) {
    if (b) {
        if (g_launches == &b->launches) g_launches = nullptr;
        cudaSetDevice(b->device);
        delete b;
    }
    return MD_OK;
}

md_status md_batch_info(const md_batch* b, int* replicas, int64_t* atoms, int* capacity, uint64_t* launches) {
    if (!b) return fail(MD_ERR_INVALID, "null batch");
    if (replicas) *replicas = b->R;
    if (atoms) *atoms = b->atoms;
    if (capacity) *capacity = b->cap;
    if (launches) *launches = b->launches;
    return MD_OK;
}

md_status md_batch_stream(md_batch* b, void** stream) {
    if (!b || !stream) return fail(MD_ERR_INVALID, "md_batch_stream: bad arguments");
    *stream = b->stream;
    return MD_OK;
}

md_status md_batch_set_force_variant(md_batch* b, int variant) {
    if (!b || variant < -1 || variant >= static_cast<int>(b->variants.size()))
        return fail(MD_ERR_INVALID, "md_batch_set_force_variant: bad arguments");
    MD_TRY(use_batch(b));
    if (variant < 0) {
        MD_TRY(b_autotune(b));
        MD_TRY(b_clear_acc(b));
    } else {
        b->variant = variant;
    }
    b->retuned = true;
    b_drop_graphs(b);
    return bsync(b);
}

md_status md_batch_force_variant(const md_batch* b, int* variant, int* count, int* particles_per_block,
                                 int* threads_per_particle) {
    if (!b) return fail(MD_ERR_INVALID, "null batch");
    if (variant) *variant = b->variant;
    if (count) *count = static_cast<int>(b->variants.size());
    if (particles_per_block) *particles_per_block = b->variants[b->variant].apb;
    if (threads_per_particle) *threads_per_particle = b->variants[b->variant].tpa;
    return MD_OK;
}

md_status md_batch_set_thermostat(md_batch* b, int thermostat, int rescale_every, double bussi_tau,
                                  const double* temperature, const uint64_t* seeds) {
    if (!b || thermostat < 0 || thermostat > 2 || (thermostat == 1 && rescale_every <= 0) ||
        (thermostat == 2 && (!(bussi_tau > 0.0) || !seeds)) || (thermostat != 0 && !temperature))
        return fail(MD_ERR_INVALID, "md_batch_set_thermostat: bad arguments");
    MD_TRY(use_batch(b));
    MD_TRY(bsync(b));
    b->opt.thermostat = thermostat;
    if (thermostat == 1) b->opt.rescale_every = rescale_every;
    if (thermostat == 2) b->opt.bussi_tau = bussi_tau;
    b->bussi_c = thermostat == 2 ? std::exp(-b->opt.dt / bussi_tau) : 0.0;  // src/Thermostat.cpp:46
    b->thermo_every = thermostat == 2 ? 1 : (thermostat == 1 ? rescale_every : 0);
    if (temperature) {
        for (int r = 0; r < b->R; ++r) b->reps_h[r].temperature = temperature[r];
        MD_CUDA(cudaMemcpyAsync(b->reps.p, b->reps_h.data(), sizeof(BRep) * b->R, cudaMemcpyHostToDevice, b->stream));
    }
    if (thermostat == 2) {  // a new BussiThermostat per replica (src/Thermostat.cpp:36-44): a fresh generator
        b->rng.clear();
        for (int r = 0; r < b->R; ++r) b->rng.emplace_back(seeds[r]);
    }
    const int chunk = b_chunk_len(b->opt, b->thermo_every);
    if (chunk != b->chunk) {
        b->chunk = chunk;
        MD_TRY(b_chunk_buffers(b));
    }
    b_drop_graphs(b);
    return bsync(b);
}

md_status md_batch_run(md_batch* b, int64_t n_steps, double* pe, double* virial, double* ke) {
    return md_batch_run_records(b, n_steps, pe, virial, ke, nullptr);
}

md_status md_batch_run_records(md_batch* b, int64_t n_steps, double* pe, double* virial, double* ke, double* inside) {
    if (!b || n_steps < 0) return fail(MD_ERR_INVALID, "md_batch_run: bad arguments");
    MD_TRY(use_batch(b));
    const int R = b->R, every = b->opt.energy_every;
    const size_t half = 2 * static_cast<size_t>(b->chunk) * R;  // draws of one chunk in h_noise
    int cur = 0;
    int64_t done = 0;
    if (n_steps > 0) b_draw(b, static_cast<int>(std::min<int64_t>(b->chunk, n_steps)), b->h_noise);
    while (done < n_steps) {
        const int len = static_cast<int>(std::min<int64_t>(b->chunk, n_steps - done));
        double* draws = b->h_noise + cur * half;
        cudaGraphExec_t g = nullptr;
        uint64_t kernels = 0;
        bool ok = false;
        for (int attempt = 0; attempt < kMaxAttempts && !ok; ++attempt) {
            if (b->opt.thermostat == 2)
                MD_CUDA(cudaMemcpyAsync(b->noise.p, draws, sizeof(double) * half, cudaMemcpyHostToDevice, b->stream));
            MD_TRY(b_snapshot(b, false));
            MD_CUDA(cudaMemsetAsync(b->flags.p, 0, sizeof(int), b->stream));
            MD_TRY(b_graph(b, len, &g, &kernels));
            MD_CUDA(cudaGraphLaunch(g, b->stream));
            b->launches += kernels;
            const int samples = every > 0 ? len / every : 0;
            if (samples > 0)
                MD_CUDA(cudaMemcpyAsync(b->h_rec, b->rec.p, sizeof(double) * kRecRows * samples * R, cudaMemcpyDeviceToHost,
                                        b->stream));
            MD_CUDA(cudaMemcpyAsync(b->h_flags, b->flags.p, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
            // the next chunk's draws are made while this one runs
            const int64_t next = done + len;
            if (attempt == 0 && next < n_steps)
                b_draw(b, static_cast<int>(std::min<int64_t>(b->chunk, n_steps - next)), b->h_noise + (1 - cur) * half);
            MD_TRY(bsync(b));
            if (b->h_flags[0] > b->cap) {
                MD_TRY(b_grow_and_restore(b, b->h_flags[0]));
                continue;
            }
            ok = true;
            for (int s = 0; s < samples; ++s) {
                const int64_t row = done / (every > 0 ? every : 1) + s;
                for (int r = 0; r < R; ++r) {
                    const double* h = b->h_rec + static_cast<size_t>(s) * kRecRows * R;
                    if (pe) pe[row * R + r] = h[r];
                    if (virial) virial[row * R + r] = h[R + r];
                    if (ke) ke[row * R + r] = h[2 * R + r];
                    if (inside) inside[row * R + r] = h[3 * R + r];
                }
            }
        }
        if (!ok) return fail(MD_ERR_CAPACITY, "neighbour row capacity could not be met");
        done += len;
        cur = 1 - cur;
        if (!b->retuned) {  // the forces of the current state, recomputed by each variant with the same bits
            b->retuned = true;
            const int before = b->variant;
            MD_TRY(b_autotune(b));
            MD_TRY(b_clear_acc(b));
            if (b->variant != before) b_drop_graphs(b);
        }
    }
    // apply the last step's pending thermostat scales
    k_b_apply_scale<<<b->tiles, kTile, 0, b->stream>>>(b->reps.p, b->tile_rep.p, b->vel.p, b->scale.p);
    MD_CHECK_LAUNCH();
    k_b_clear_scale<<<per_replica(b, kThreads), kThreads, 0, b->stream>>>(R, b->scale.p);
    MD_CHECK_LAUNCH();
    return bsync(b);
}

// Potential energy, virial, inside-cutoff count and kinetic energy of every replica's current state
md_status md_batch_energy(md_batch* b, double* pe, double* virial, double* ke, double* inside) {
    if (!b) return fail(MD_ERR_INVALID, "null batch");
    MD_TRY(use_batch(b));
    MD_TRY(b_clear_acc(b));
    MD_TRY(b_forces(b, b->variant, false, true));
    MD_TRY(b_observables(b, b->tmp_pe.p, b->tmp_w.p, b->ke.p));
    const size_t R = b->R;
    std::vector<double> hp(R), hw(R), hk(R);
    std::vector<unsigned long long> hi(R);
    MD_CUDA(cudaMemcpyAsync(hp.data(), b->tmp_pe.p, sizeof(double) * R, cudaMemcpyDeviceToHost, b->stream));
    MD_CUDA(cudaMemcpyAsync(hw.data(), b->tmp_w.p, sizeof(double) * R, cudaMemcpyDeviceToHost, b->stream));
    MD_CUDA(cudaMemcpyAsync(hk.data(), b->ke.p, sizeof(double) * R, cudaMemcpyDeviceToHost, b->stream));
    MD_CUDA(cudaMemcpyAsync(hi.data(), b->inside.p, sizeof(unsigned long long) * R, cudaMemcpyDeviceToHost, b->stream));
    MD_TRY(bsync(b));
    for (size_t r = 0; r < R; ++r) {
        if (pe) pe[r] = hp[r];
        if (virial) virial[r] = hw[r];
        if (ke) ke[r] = hk[r];
        if (inside) inside[r] = static_cast<double>(hi[r]);
    }
    return MD_OK;
}

md_status md_batch_download(md_batch* b, int replica, double* pos4, double* vel3, double* force3, double* mass,
                            uint64_t* ids) {
    if (!b || replica < 0 || replica >= b->R) return fail(MD_ERR_INVALID, "md_batch_download: bad arguments");
    MD_TRY(use_batch(b));
    const BRep& d = b->reps_h[replica];
    const size_t n = static_cast<size_t>(d.n);
    if (pos4) MD_CUDA(cudaMemcpyAsync(pos4, b->pos.p + d.off, sizeof(double4) * n, cudaMemcpyDeviceToHost, b->stream));
    for (int k = 0; k < 3; ++k) {
        const size_t src = 3 * static_cast<size_t>(d.off) + static_cast<size_t>(k) * d.np;
        if (vel3) MD_CUDA(cudaMemcpyAsync(vel3 + k * n, b->vel.p + src, sizeof(double) * n, cudaMemcpyDeviceToHost, b->stream));
        if (force3)
            MD_CUDA(cudaMemcpyAsync(force3 + k * n, b->force.p + src, sizeof(double) * n, cudaMemcpyDeviceToHost, b->stream));
    }
    if (mass) MD_CUDA(cudaMemcpyAsync(mass, b->mass.p + d.off, sizeof(double) * n, cudaMemcpyDeviceToHost, b->stream));
    if (ids) MD_CUDA(cudaMemcpyAsync(ids, b->ids.p + d.off, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, b->stream));
    return bsync(b);
}

md_status md_batch_state_hash(md_batch* b, uint64_t* hashes) {
    if (!b || !hashes) return fail(MD_ERR_INVALID, "md_batch_state_hash: bad arguments");
    for (int r = 0; r < b->R; ++r) {
        const size_t n = static_cast<size_t>(b->reps_h[r].n);
        std::vector<double> pos(4 * n), vel(3 * n);
        MD_TRY(md_batch_download(b, r, pos.data(), vel.data(), nullptr, nullptr, nullptr));
        // FNV-1a over (x, vx, y, vy, z, vz) per particle (src/System.cpp:85-105)
        uint64_t h = 14695981039346656037ull;
        auto mix = [&h](double v) {
            uint64_t bits;
            std::memcpy(&bits, &v, 8);
            for (unsigned k = 0; k < 8; ++k) {
                h ^= (bits >> (8u * k)) & 0xffu;
                h *= 1099511628211ull;
            }
        };
        for (size_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) {
                mix(pos[4 * i + k]);
                mix(vel[k * n + i]);
            }
        hashes[r] = h;
    }
    return MD_OK;
}

md_status md_batch_rebuilds(md_batch* b, uint64_t* rebuilds) {
    if (!b || !rebuilds) return fail(MD_ERR_INVALID, "md_batch_rebuilds: bad arguments");
    MD_TRY(use_batch(b));
    MD_CUDA(cudaMemcpyAsync(rebuilds, b->rebuilds.p, sizeof(unsigned long long) * b->R, cudaMemcpyDeviceToHost, b->stream));
    return bsync(b);
}

// Average duration of the list force kernel alone (no kick, no energy) over `reps` launches, CUDA events on
// the batch's stream
md_status md_batch_time_forces(md_batch* b, int reps, double* ms) {
    if (!b || reps <= 0 || !ms) return fail(MD_ERR_INVALID, "md_batch_time_forces: bad arguments");
    MD_TRY(use_batch(b));
    cudaEvent_t e0, e1;
    MD_CUDA(cudaEventCreate(&e0));
    MD_CUDA(cudaEventCreate(&e1));
    md_status st = b_forces(b, b->variant, false, false);
    if (st == MD_OK) cudaEventRecord(e0, b->stream);
    for (int k = 0; k < reps && st == MD_OK; ++k) st = b_forces(b, b->variant, false, false);
    if (st == MD_OK) cudaEventRecord(e1, b->stream);
    float t = 0.f;
    if (st == MD_OK && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MD_TRY(st);
    MD_TRY(b_clear_acc(b));
    *ms = static_cast<double>(t) / reps;
    return bsync(b);
}

}  // extern "C"
