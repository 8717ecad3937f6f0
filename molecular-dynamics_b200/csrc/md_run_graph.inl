// md_run as CUDA graphs: the float precisions on a tiled list. Included by md_abi.cu after md_abi_float.inl.
//
// A run is cut into chunks of up to s->graph_chunk steps; each chunk is one CUDA graph, cached by everything it
// records (buffer addresses, sizes, constants and the chunk's step pattern). A step in a graph is the host loop's
// step (run_steps) with the rebuild decision moved to the device: a one-thread kernel turns the half-skin flag
// of the last drift into the condition of an IF node whose body is the list rebuild, enqueued by the same
// kernels as the host path (cell sort, reorder, frames, tiled build; MD_PREC_FX32's near-first rows and the
// fixed-point frames). So a chunk needs one host synchronisation instead of one per step.
//
// Addresses: the graph's kernels are recorded with the buffers' addresses, so inside a graph nothing may change
// which buffer holds what. The rebuild reorders into the spare arrays and copies back (the host path swaps
// instead), and every chunk starts and ends with each double-buffered array (positions, velocities, forces,
// masses, ids, float and fixed-point frames) in its canonical buffer: the fused drift alternates positions and
// frames between the two buffers step by step, so a chunk with an odd number of fused steps ends with one copy.
//
// Capacity: a rebuild whose rows outgrow the capacity, or whose cells outgrow the shared-memory tile recorded in
// the graph, sets an error flag (rows are never written out of bounds). The chunk then starts again on the host
// path from a snapshot the graph took at its start (positions, velocities, forces, masses, ids, the list's
// reference positions, the stale flag and the g(r) histogram): the list of the chunk's start is rebuilt from the
// reference positions (particles already in cell order, so the reorder is the identity and the rows are the
// same), then the host grows what it must. Either way the trajectory is the host path's, bit for bit.

namespace {

constexpr int kGraphMaxSteps = 1024;  // steps per chunk graph at most

struct RunStep {
    bool drifted_in = false;  // the previous step's force kernel made this step's kick and drift
    bool fuse_out = false;    // this step's force kernel makes the next step's kick and drift
    int thermo = 0;           // 0 none, 1 rescale, 2 Bussi
    double target = 0.0;      // rescale target temperature
    bool rdf = false;         // g(r) sample after the step
};

bool float_precision(int p) {
    return p == MD_PREC_FP32FX || p == MD_PREC_FP32 || p == MD_PREC_FX64 || p == MD_PREC_FX32;
}

// Step k (0-based) of a run of n_steps, as run_steps decides it (fusable: the float precisions, whose force kernel
// can make the next step's kick and drift)
RunStep plan_step(const md_run_options& o, int64_t k, int64_t n_steps, bool drifted_in, bool fusable) {
    RunStep r;
    const int64_t step = o.first_step + k;
    r.drifted_in = drifted_in;
    const bool rescale = o.thermostat == 1 && o.rescale_every > 0 && step % o.rescale_every == 0;
    r.thermo = rescale ? 1 : (o.thermostat == 2 ? 2 : 0);
    r.target = rescale ? (step <= o.melt_until ? o.melt_temperature : o.rescale_temperature) : 0.0;
    r.rdf = o.rdf && o.rdf_every > 0 && step % o.rdf_every == 0;
    r.fuse_out = fusable && k + 1 < n_steps && r.thermo == 0 && !r.rdf;
    return r;
}

// The step's (PE, virial) into rec[0..1] on the stream where they end (FP64: the chain stream of its ordered sums),
// as run_steps records them
md_status record_energy(md_forcefield* ff, md_system* s, double* rec, bool want_energy) {
    if (!want_energy) return MD_OK;
    const cudaStream_t es = energy_stream(ff, s);
    MD_CUDA(cudaMemcpyAsync(rec, ff->out.p, 2 * sizeof(double), cudaMemcpyDeviceToDevice, es));
    if (es != s->stream) MD_CUDA(cudaEventRecord(ff->ev_done, es));  // the join covers the copy too
    return MD_OK;
}

// MD_PREC_FP64 runs as graphs up to this many particles. Measured on the B200 (microseconds per step with energies
// recorded, graph / host loop): 2,048: 79 / 99; 32,000: 87 / 105; 256,000: 293 / 318; 4,000,000: 3,253 / 2,410.
// For a large list the ordered energy sums (a 1.1 ms chain at 4M) overlap the next steps on their own streams,
// which a graph's branches did not match.
constexpr int64_t kFp64GraphMaxParticles = 1'000'000;

// Can md_run use graphs for this call? (a tiled list built for this system; the tiled build is the one the device
// rebuild enqueues)
bool graph_mode_ok(const md_system* s, const md_forcefield* ff, const md_nlist* nl, int64_t n_steps) {
    const bool precision = float_precision(ff->precision) ||
                           (ff->precision == MD_PREC_FP64 && s->n <= kFp64GraphMaxParticles);
    return s->graph_chunk > 0 && n_steps > 0 && s->n > 0 && precision && nlist_current(nl, s) && nl->use_cells &&
           nl->use_tiles && nl->build_pin != 0;
}

// Live data of a double-buffered array into its canonical buffer (recorded by the graphs); count elements
template <typename T>
md_status to_canonical(DevBuf<T>& cur, DevBuf<T>& spare, void*& canon, size_t count, cudaStream_t st) {
    if (!cur.p) return MD_OK;
    if (canon != cur.p && canon != spare.p) canon = cur.p;  // first use, or a buffer was reallocated
    if (cur.p != canon) {
        MD_CUDA(cudaMemcpyAsync(spare.p, cur.p, sizeof(T) * count, cudaMemcpyDeviceToDevice, st));
        swap_buffers(cur, spare);
    }
    return MD_OK;
}

md_status normalize_buffers(md_system* s, md_nlist* nl) {
    const size_t n = static_cast<size_t>(s->n);
    cudaStream_t st = s->stream;
    MD_TRY(to_canonical(s->pos, s->pos2, s->canon[0], n, st));
    MD_TRY(to_canonical(s->vel, s->vel2, s->canon[1], 3 * n, st));
    MD_TRY(to_canonical(s->force, s->force2, s->canon[2], 3 * n, st));
    MD_TRY(to_canonical(s->mass, s->mass2, s->canon[3], n, st));
    MD_TRY(to_canonical(s->ids, s->ids2, s->canon[4], n, st));
    MD_TRY(to_canonical(nl->frames, nl->frames2, s->canon[5], n + 1, st));
    MD_TRY(to_canonical(nl->iframes, nl->iframes2, s->canon[6], n, st));
    return MD_OK;
}

// Everything a chunk graph uses is allocated, tuned and current before capture (no allocation, host read or
// tuning may happen while a stream is captured)
md_status graph_prepare_buffers(md_system* s, md_forcefield* ff, md_nlist* nl, const md_run_options& o) {
    const int n = static_cast<int>(s->n);
    const size_t C = static_cast<size_t>(s->graph_chunk);
    MD_CUDA(s->pos2.reserve(n));
    MD_CUDA(s->vel2.reserve(3 * static_cast<size_t>(n)));
    MD_CUDA(s->force2.reserve(3 * static_cast<size_t>(n)));
    MD_CUDA(s->mass2.reserve(n));
    MD_CUDA(s->ids2.reserve(n));
    MD_CUDA(nl->frames.reserve(static_cast<size_t>(n) + 1));
    MD_CUDA(nl->frames2.reserve(static_cast<size_t>(n) + 1));
    MD_CUDA(nl->iframes.reserve(n));
    MD_CUDA(nl->iframes2.reserve(n));
    MD_CUDA(ff->out.reserve(4));
    MD_CUDA(ff->inside_count.reserve(1));
    MD_CUDA(ff->fx_acc.reserve(4));
    MD_CUDA(s->graph_state.reserve(2));
    MD_CUDA(s->chunk_rec.reserve(3 * C));
    MD_CUDA(s->chunk_noise.reserve(2 * C));
    MD_CUDA(s->snap_pos.reserve(n));
    MD_CUDA(s->snap_ref.reserve(n));
    MD_CUDA(s->snap_vel.reserve(3 * static_cast<size_t>(n)));
    MD_CUDA(s->snap_force.reserve(3 * static_cast<size_t>(n)));
    MD_CUDA(s->snap_mass.reserve(n));
    MD_CUDA(s->snap_ids.reserve(n));
    MD_CUDA(s->snap_flag.reserve(1));
    if (!s->body_stream) MD_CUDA(cudaStreamCreateWithFlags(&s->body_stream, cudaStreamNonBlocking));
    if (o.rdf) {
        if (o.rdf->device < 0) {
            o.rdf->device = s->device;
            MD_CUDA(o.rdf->hist.reserve(o.rdf->bins));
            MD_CUDA(cudaMemsetAsync(o.rdf->hist.p, 0, sizeof(unsigned long long) * o.rdf->bins, s->stream));
        }
        MD_CUDA(s->snap_hist.reserve(o.rdf->bins));
    }
    if (ff->precision == MD_PREC_FX32) MD_TRY(ensure_near_first(ff, s, nl));
    if (ff->precision == MD_PREC_FP64) {
        // the energy records of the lists a graph builds: a quarter more than the current list's pairs (a chunk
        // whose rebuild outgrows them reruns on the host path, which grows them); the kinetic-energy blocks
        MD_TRY(ensure_pairs(nl));
        if (!ff->side) MD_TRY(energy_streams(ff));
        MD_TRY(energy_quiesce(ff));
        const long long pairs = static_cast<long long>(nl->pairs);
        MD_TRY(reserve_energy_records(ff, pairs + pairs / 4 + kChunk));
        MD_CUDA(s->ke_blocks.reserve(static_cast<size_t>((n + kChunk - 1) / kChunk)));
    }
    // the resident grids of the force kernels that size their launch by occupancy, known before any capture
    int sms = 0;
    MD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
    auto grid = [&](auto kernel, unsigned& g) -> md_status {
        if (g == 0) {
            int per_sm = 0;
            MD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0));
            g = static_cast<unsigned>(std::max(1, sms * per_sm));
        }
        return MD_OK;
    };
    MD_TRY(grid(k_force_fp32_resident<false, false>, s->fp32_resident[0][0]));
    MD_TRY(grid(k_force_fp32_resident<false, true>, s->fp32_resident[0][1]));
    MD_TRY(grid(k_force_fp32_resident<true, false>, s->fp32_resident[1][0]));
    MD_TRY(grid(k_force_fp32_resident<true, true>, s->fp32_resident[1][1]));
    MD_TRY(grid(k_force_fx32<false>, s->fx32_resident[0]));
    MD_TRY(grid(k_force_fx32<true>, s->fx32_resident[1]));
    return MD_OK;
}

// The tile geometry recorded in a graph: the host's, with room for cells that fill up at later rebuilds
TileGeom graph_geometry(const md_system* s, const md_nlist* nl) {
    TileGeom g = nl->tiles_geom;
    // a quarter more, rounded up to 256 slots (so a run's graphs survive small changes of the host's bound)
    g.max_staged = std::min(((g.max_staged + g.max_staged / 4 + 64 + 255) / 256) * 256, 12000);
    return g;
}

// NeighbourList::build on the device without host reads (the graph's rebuild body): the same kernels as
// nlist_build, the reorder copied back into the system's own arrays, the result checked on the device
md_status device_rebuild_async(md_system* s, md_forcefield* ff, md_nlist* nl, const TileGeom& tg) {
    const int n = static_cast<int>(s->n);
    CellGrid& g = nl->grid;
    cudaStream_t st = s->stream;
    k_zero_ints<<<std::min(blocks_for(g.ncells, kThreads), 148u * 8u), kThreads, 0, st>>>(g.count.p, g.ncells,
                                                                                       g.cursor.p, g.ncells);
    MD_CHECK_LAUNCH();
    k_cell_assign<<<blocks_for(n, kThreads), kThreads, 0, st>>>(s->pos.p, n, g.ncps / s->box.L, g.ncps, g.cell_of.p,
                                                                g.count.p);
    MD_CHECK_LAUNCH();
    exclusive_scan<int, int>(g.count.p, g.ncells, g.start.p, g.tiles.p, st);
    MD_CHECK_SCAN();
    k_cell_scatter<<<blocks_for(n, kThreads), kThreads, 0, st>>>(g.cell_of.p, n, g.start.p, g.cursor.p, g.bucket.p);
    MD_CHECK_LAUNCH();
    k_cell_rank<<<blocks_for(static_cast<long long>(g.ncells) * 32, kThreads), kThreads, 0, st>>>(
        g.start.p, g.ncells, g.bucket.p, g.order.p);
    MD_CHECK_LAUNCH();
    k_permute<<<blocks_for(n, kThreads), kThreads, 0, st>>>(g.order.p, n, s->pos.p, s->vel.p, s->force.p, s->mass.p,
                                                            s->ids.p, s->pos2.p, s->vel2.p, s->force2.p, s->mass2.p,
                                                            s->ids2.p, g.cell_of.p, nl->cell_sorted.p, nl->ref_pos.p);
    MD_CHECK_LAUNCH();
    k_copy_back<<<blocks_for(n, kThreads), kThreads, 0, st>>>(n, s->pos2.p, s->vel2.p, s->force2.p, s->mass2.p,
                                                              s->ids2.p, s->pos.p, s->vel.p, s->force.p, s->mass.p,
                                                              s->ids.p);
    MD_CHECK_LAUNCH();
    const double cell = s->box.L / g.ncps;
    k_frames<<<blocks_for(n + 1, kThreads), kThreads, 0, st>>>(s->pos.p, n, nl->cell_sorted.p, g.ncps, cell, s->box,
                                                               nl->frames.p);
    MD_CHECK_LAUNCH();
    const double margin = 1e-5 * nl->rl2 + 1e-4;
    const BuildParams bp{nl->rl2, static_cast<float>(nl->rl2 - margin), static_cast<float>(nl->rl2 + margin), nl->cap,
                         static_cast<uint32_t>(n)};
    const size_t smem = sizeof(float4) * tg.max_staged;
    MD_CUDA(allow_smem(k_nlist_build_tile, smem));
    k_nlist_build_tile<<<tile_blocks(tg), kTileThreads, smem, st>>>(nl->frames.p, s->pos.p, g.start.p,
                                                                    nl->cell_sorted.p, tg, bp, cell_offsets(nl, s),
                                                                    nl->rows.p, nl->counts.p, nl->flags.p + 1);
    MD_CHECK_LAUNCH();
    k_build_done<<<1, 1, 0, st>>>(nl->flags.p + 1, nl->cap, s->graph_state.p, (s->graph_flags & MD_GRAPH_TEST_RERUN) != 0);
    MD_CHECK_LAUNCH();
    if (ff->precision == MD_PREC_FP64) {  // the pair offsets of the energy records, and their count against the buffers
        k_own_counts<<<blocks_for(n, kThreads), kThreads, 0, st>>>(nl->counts.p, n, nl->tmp_counts.p);
        MD_CHECK_LAUNCH();
        exclusive_scan<int, long long>(nl->tmp_counts.p, n, nl->half_off.p, nl->tiles.p, st);
        MD_CHECK_SCAN();
        const long long cap = static_cast<long long>(std::min(ff->pair_r2[0].count, ff->pair_r2[1].count) / 2);
        k_pairs_fit<<<1, 1, 0, st>>>(nl->half_off.p + n, cap, s->graph_state.p);
        MD_CHECK_LAUNCH();
    }
    if (ff->precision == MD_PREC_FX32)  // the rows just built, split (the float frames are the build's)
        MD_TRY(split_rows_async(s, nl, nl->frames.p, static_cast<float>(nl->nf_near2), st));
    if (ff->precision == MD_PREC_FX64 || ff->precision == MD_PREC_FX32) {
        k_frames_fixed<<<blocks_for(n, kThreads), kThreads, 0, st>>>(s->pos.p, n, nl->cell_sorted.p, g.ncps, cell,
                                                                     s->box, nl->iframes.p);
        MD_CHECK_LAUNCH();
    }
    return MD_OK;
}

// A key of everything a chunk graph records
std::string graph_key(const md_system* s, const md_forcefield* ff, const md_nlist* nl, const md_run_options& o,
                      const std::vector<RunStep>& steps, double dt, bool want_energy, bool want_ke, double bussi_c,
                      const TileGeom& tg) {
    std::string k;
    char buf[96];
    auto ptr = [&](const void* p) {
        std::snprintf(buf, sizeof buf, "%p,", p);
        k += buf;
    };
    auto num = [&](double v) {
        std::snprintf(buf, sizeof buf, "%a,", v);
        k += buf;
    };
    for (const void* p : {static_cast<const void*>(s->pos.p), static_cast<const void*>(s->pos2.p),
                          static_cast<const void*>(s->vel.p), static_cast<const void*>(s->vel2.p),
                          static_cast<const void*>(s->force.p), static_cast<const void*>(s->force2.p),
                          static_cast<const void*>(s->mass.p), static_cast<const void*>(s->mass2.p),
                          static_cast<const void*>(s->ids.p), static_cast<const void*>(s->ids2.p),
                          static_cast<const void*>(s->scal.p), static_cast<const void*>(s->graph_state.p),
                          static_cast<const void*>(s->chunk_rec.p), static_cast<const void*>(s->chunk_noise.p),
                          static_cast<const void*>(s->snap_pos.p), static_cast<const void*>(s->snap_ref.p),
                          static_cast<const void*>(s->snap_vel.p), static_cast<const void*>(s->snap_force.p),
                          static_cast<const void*>(s->snap_mass.p), static_cast<const void*>(s->snap_ids.p),
                          static_cast<const void*>(s->snap_flag.p), static_cast<const void*>(s->snap_hist.p),
                          static_cast<const void*>(nl->frames.p), static_cast<const void*>(nl->frames2.p),
                          static_cast<const void*>(nl->iframes.p), static_cast<const void*>(nl->iframes2.p),
                          static_cast<const void*>(nl->rows.p), static_cast<const void*>(nl->counts.p),
                          static_cast<const void*>(nl->rows_nf.p), static_cast<const void*>(nl->counts_nf.p),
                          static_cast<const void*>(nl->cell_sorted.p), static_cast<const void*>(nl->ref_pos.p),
                          static_cast<const void*>(nl->flags.p), static_cast<const void*>(nl->grid.cell_of.p),
                          static_cast<const void*>(nl->grid.count.p), static_cast<const void*>(nl->grid.start.p),
                          static_cast<const void*>(nl->grid.cursor.p), static_cast<const void*>(nl->grid.bucket.p),
                          static_cast<const void*>(nl->grid.order.p), static_cast<const void*>(nl->grid.tiles.p),
                          static_cast<const void*>(ff->fx_acc.p), static_cast<const void*>(ff->out.p),
                          static_cast<const void*>(ff->inside_count.p), static_cast<const void*>(ff->pair_r2[0].p),
                          static_cast<const void*>(ff->pair_r2[1].p), static_cast<const void*>(ff->eblocks[0].p),
                          static_cast<const void*>(ff->eblocks[1].p), static_cast<const void*>(s->ke_blocks.p),
                          static_cast<const void*>(ff->epairs.p), static_cast<const void*>(ff->enblocks.p),
                          static_cast<const void*>(nl->half_off.p), static_cast<const void*>(nl->tmp_counts.p),
                          static_cast<const void*>(nl->tiles.p),
                          static_cast<const void*>(o.rdf ? o.rdf->hist.p : nullptr)})
        ptr(p);
    for (double v : {static_cast<double>(s->n), s->box.L, static_cast<double>(nl->cap), static_cast<double>(tg.kk),
                     static_cast<double>(tg.nseg), static_cast<double>(tg.max_staged), static_cast<double>(tg.ncps),
                     static_cast<double>(nl->variant[ff->precision]), static_cast<double>(ff->precision), ff->eps,
                     ff->sigma, ff->rc, nl->rl2, nl->max_disp2, nl->nf_near2, dt, want_energy ? 1.0 : 0.0,
                     want_ke ? 1.0 : 0.0, bussi_c, o.bussi_temperature, s->profile ? 1.0 : 0.0,
                     static_cast<double>(s->graph_chunk), o.rdf ? o.rdf->rmax : 0.0,
                     static_cast<double>(o.rdf ? o.rdf->bins : 0), static_cast<double>(ff->serial),
                     static_cast<double>(nl->serial), static_cast<double>(ff->pair_r2[0].count),
                     static_cast<double>(ff->pair_r2[1].count)})
        num(v);
    for (const RunStep& r : steps) {
        std::snprintf(buf, sizeof buf, "%d%d%d%d", r.drifted_in, r.fuse_out, r.thermo, r.rdf);
        k += buf;
        if (r.thermo == 1) num(r.target);
        k += ';';
    }
    return k;
}

// One step of a chunk, captured: run_steps' step with the rebuild in a conditional node
md_status graph_step(md_system* s, md_forcefield* ff, md_nlist* nl, const md_run_options& o, const RunStep& r, int k,
                     double dt, bool want_energy, bool want_ke, double bussi_c, cudaGraph_t graph, const TileGeom& tg,
                     uint64_t* body_kernels) {
    const bool float_frames =
        ff->precision == MD_PREC_FP32FX || ff->precision == MD_PREC_FP32 || ff->precision == MD_PREC_FX32;
    if (!r.drifted_in) MD_TRY(kick_drift_async(s, nl, dt, true, float_frames));
    cudaGraphConditionalHandle h;
    MD_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault));
    k_set_rebuild<<<1, 1, 0, s->stream>>>(h, nl->flags.p);
    MD_CHECK_LAUNCH();
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    MD_CUDA(cudaStreamGetCaptureInfo(s->stream, &cs, nullptr, &cg, &deps, &nd));
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeIf;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    MD_CUDA(cudaGraphAddNode(&node, cg, deps, nd, &p));
    MD_CUDA(cudaStreamUpdateCaptureDependencies(s->stream, &node, 1, cudaStreamSetCaptureDependencies));
    {
        cudaGraph_t body = p.conditional.phGraph_out[0];
        const cudaStream_t main = s->stream;
        uint64_t* saved = g_launches;
        uint64_t count = 0;
        g_launches = &count;
        MD_CUDA(cudaStreamBeginCaptureToGraph(s->body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        s->stream = s->body_stream;
        const md_status st = device_rebuild_async(s, ff, nl, tg);
        s->stream = main;
        g_launches = saved;
        const cudaError_t e = cudaStreamEndCapture(s->body_stream, &body);
        MD_TRY(st);
        MD_CUDA(e);
        *body_kernels = count;
    }
    // the frames are current after a fused drift or a rebuild body; after this step's own drift the fixed-point
    // frames are made again (the float frames were written by the drift)
    bool fused_ke = false;
    MD_TRY(forces_list_async(ff, s, nl, want_energy, dt, true, &fused_ke, r.fuse_out, r.drifted_in));
    double* rec = s->chunk_rec.p + 3 * static_cast<size_t>(k);
    MD_TRY(record_energy(ff, s, rec, want_energy));
    bool ke_current = fused_ke;
    if (r.thermo) {
        if (!ke_current) MD_TRY(kinetic_async(s));
        if (r.thermo == 1) {
            k_rescale_factor<<<1, 1, 0, s->stream>>>(s->scal.p + kScalKE, dof_of(s->n), r.target, s->scal.p + kScalFactor);
        } else {
            const double* noise = s->chunk_noise.p;
            k_bussi_factor<<<1, 1, 0, s->stream>>>(s->scal.p + kScalKE, dof_of(s->n), o.bussi_temperature, bussi_c,
                                                   noise + k, noise + s->graph_chunk + k, s->scal.p + kScalFactor);
        }
        MD_CHECK_LAUNCH();
        MD_TRY(scale_async(s));
        ke_current = false;
    }
    if (r.rdf) MD_TRY(rdf_kernel_async(o.rdf, s, nl));
    if (want_ke) {
        if (!ke_current) MD_TRY(ff->precision == MD_PREC_FP64 ? kinetic_async(s) : kinetic_fixed_async(s, ff));
        MD_CUDA(cudaMemcpyAsync(rec + 2, s->scal.p + kScalKE, sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
    }
    return MD_OK;
}

// The graph of one chunk (captured once per key)
md_status chunk_graph(md_system* s, md_forcefield* ff, md_nlist* nl, const md_run_options& o,
                      const std::vector<RunStep>& steps, double dt, bool want_energy, bool want_ke, double bussi_c,
                      RunGraph** out) {
    const TileGeom tg = graph_geometry(s, nl);
    const std::string key = graph_key(s, ff, nl, o, steps, dt, want_energy, want_ke, bussi_c, tg);
    auto it = s->graphs.find(key);
    if (it != s->graphs.end()) {
        *out = &it->second;
        return MD_OK;
    }
    if (s->graphs.size() >= 32) drop_run_graphs(s);
    const int n = static_cast<int>(s->n);
    const size_t N = static_cast<size_t>(n);
    RunGraph rg;
    // what a capture may not do: opt the tile kernels in to the recorded tile's shared memory, create the
    // profiling events (two per step)
    const size_t build_smem = sizeof(float4) * tg.max_staged, tile_smem = sizeof(float4) * (tg.max_staged + 1);
    MD_CUDA(allow_smem(k_nlist_build_tile, build_smem));
    MD_CUDA(allow_smem(k_force_fp32_tile<true, true>, tile_smem));
    MD_CUDA(allow_smem(k_force_fp32_tile<true, false>, tile_smem));
    MD_CUDA(allow_smem(k_force_fp32_tile<false, true>, tile_smem));
    MD_CUDA(allow_smem(k_force_fp32_tile<false, false>, tile_smem));
    MD_CUDA(allow_smem(k_force_fp64_tile<true>, sizeof(double4) * tg.max_staged));
    MD_CUDA(allow_smem(k_force_fp64_tile<false>, sizeof(double4) * tg.max_staged));
    // FP64: the capture starts with no energy sums queued and the records' first buffers (energy_quiesce)
    MD_TRY(energy_quiesce(ff));
    if (s->profile) {
        rg.prof.resize(2 * steps.size());
        for (cudaEvent_t& ev : rg.prof) MD_CUDA(cudaEventCreate(&ev));
    }
    cudaGraph_t graph = nullptr;
    MD_CUDA(cudaGraphCreate(&graph, 0));
    uint64_t* saved = g_launches;
    uint64_t count = 0, body = 0;
    g_launches = &count;
    const TileGeom host_geom = nl->tiles_geom;
    nl->tiles_geom = tg;  // the tile force kernel, if it is the one in use, records the same bound as the build
    std::vector<cudaEvent_t>* saved_prof = g_capture_prof;
    g_capture_prof = s->profile ? &rg.prof : nullptr;
    g_capture_prof_next = 0;
    g_graph_overflow = s->graph_state.p + 1;
    g_capturing = true;
    md_status st = MD_OK;
    cudaError_t e = cudaStreamBeginCaptureToGraph(s->stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        auto cp = [&](void* dst, const void* src, size_t bytes) {
            if (st == MD_OK && bytes) {
                const cudaError_t c = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s->stream);
                if (c != cudaSuccess) st = fail(MD_ERR_CUDA, std::string("graph snapshot: ") + cudaGetErrorString(c));
            }
        };
        // prologue: clear the device counters and take the snapshot the host restarts from on an overflow
        if (cudaMemsetAsync(s->graph_state.p, 0, 2 * sizeof(int), s->stream) != cudaSuccess)
            st = fail(MD_ERR_CUDA, "graph state reset");
        cp(s->snap_pos.p, s->pos.p, sizeof(double4) * N);
        cp(s->snap_vel.p, s->vel.p, sizeof(double) * 3 * N);
        cp(s->snap_force.p, s->force.p, sizeof(double) * 3 * N);
        cp(s->snap_mass.p, s->mass.p, sizeof(double) * N);
        cp(s->snap_ids.p, s->ids.p, sizeof(uint64_t) * N);
        cp(s->snap_ref.p, nl->ref_pos.p, sizeof(double4) * N);
        cp(s->snap_flag.p, nl->flags.p, sizeof(int));
        bool rdf = false;
        for (const RunStep& r : steps) rdf |= r.rdf;
        if (rdf) cp(s->snap_hist.p, o.rdf->hist.p, sizeof(unsigned long long) * o.rdf->bins);
        for (size_t k = 0; k < steps.size() && st == MD_OK; ++k) {
            uint64_t b = 0;
            st = graph_step(s, ff, nl, o, steps[k], static_cast<int>(k), dt, want_energy, want_ke, bussi_c, graph, tg, &b);
            body = b;
            rg.rdf_samples += steps[k].rdf ? 1 : 0;
        }
        // epilogue: positions and frames back into their canonical buffers
        if (st == MD_OK && s->pos.p != s->canon[0]) {
            cp(s->pos2.p, s->pos.p, sizeof(double4) * N);
            swap_buffers(s->pos, s->pos2);
        }
        if (st == MD_OK && nl->frames.p != s->canon[5]) {
            cp(nl->frames2.p, nl->frames.p, sizeof(float4) * (N + 1));
            swap_buffers(nl->frames, nl->frames2);
        }
        if (st == MD_OK && nl->iframes.p != s->canon[6]) {
            cp(nl->iframes2.p, nl->iframes.p, sizeof(int4) * N);
            swap_buffers(nl->iframes, nl->iframes2);
        }
        // FP64: the energy sums' streams joined back into the graph's end
        for (int b = 0; b < 2 && st == MD_OK; ++b) {
            if (ff->read_pending[b] && cudaStreamWaitEvent(s->stream, ff->ev_read[b], 0) != cudaSuccess)
                st = fail(MD_ERR_CUDA, "graph join of the block sums");
            if (ff->chain_pending[b] && cudaStreamWaitEvent(s->stream, ff->ev_chain[b], 0) != cudaSuccess)
                st = fail(MD_ERR_CUDA, "graph join of the ordered sums");
        }
        if (st == MD_OK && ff->side_pending && cudaStreamWaitEvent(s->stream, ff->ev_done, 0) != cudaSuccess)
            st = fail(MD_ERR_CUDA, "graph join of the energy records");
        e = cudaStreamEndCapture(s->stream, &graph);
    }
    // nothing the capture recorded has run: the host's record of queued sums starts afresh
    const md_status eq = energy_quiesce(ff);
    if (st == MD_OK) st = eq;
    g_capture_prof = saved_prof;
    g_graph_overflow = nullptr;
    g_capturing = false;
    g_launches = saved;
    nl->tiles_geom = host_geom;
    if (st != MD_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        for (cudaEvent_t ev : rg.prof) cudaEventDestroy(ev);
        cudaGetLastError();
        if (st != MD_OK) return st;
        return fail(MD_ERR_CUDA, std::string("md_run graph capture: ") + cudaGetErrorString(e));
    }
    // per-node priorities: the FP64 energy sums' kernels carry the highest (launch_priority), as on their streams
    const cudaError_t ei = cudaGraphInstantiate(&rg.exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        for (cudaEvent_t ev : rg.prof) cudaEventDestroy(ev);
        return fail(MD_ERR_CUDA, std::string("md_run graph instantiate: ") + cudaGetErrorString(ei));
    }
    rg.kernels = count;
    rg.body_kernels = body;
    auto ins = s->graphs.emplace(key, std::move(rg));
    *out = &ins.first->second;
    return MD_OK;
}

// The chunks of a run: [begin, end) step ranges of at most graph_chunk steps
std::vector<std::pair<int64_t, int64_t>> run_chunks(const md_system* s, int64_t k0, int64_t n_steps) {
    std::vector<std::pair<int64_t, int64_t>> c;
    const int64_t C = std::min<int64_t>(s->graph_chunk, kGraphMaxSteps);
    for (int64_t b = k0; b < n_steps; b += C) c.emplace_back(b, std::min(n_steps, b + C));
    return c;
}

std::vector<RunStep> chunk_steps(const md_run_options& o, int64_t b, int64_t e, int64_t n_steps, bool fusable) {
    std::vector<RunStep> v;
    bool drifted = false;
    for (int64_t k = 0; k < e; ++k) {
        const RunStep r = plan_step(o, k, n_steps, drifted, fusable);
        if (k >= b) v.push_back(r);
        drifted = r.fuse_out;
    }
    return v;
}

// md_run_prepare: capture the graphs a run with these arguments would launch
md_status graph_prepare(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps,
                        const md_run_options& o, bool want_energy, bool want_ke) {
    MD_TRY(graph_prepare_buffers(s, ff, nl, o));
    MD_TRY(normalize_buffers(s, nl));
    const double bussi_c = o.thermostat == 2 ? std::exp(-dt / o.bussi_tau) : 0.0;
    for (const auto& c : run_chunks(s, nl->variant[ff->precision] < 0 ? 1 : 0, n_steps)) {
        RunGraph* g = nullptr;
        MD_TRY(chunk_graph(s, ff, nl, o, chunk_steps(o, c.first, c.second, n_steps, float_precision(ff->precision)), dt,
                           want_energy, want_ke, bussi_c, &g));
    }
    return MD_OK;
}

// The host loop's step k of a run (run_steps), used to run a chunk again after an overflow in its graph
md_status host_step(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps, const md_run_options& o,
                    int64_t k, bool drifted_in, bool want_energy, bool want_ke, const double* noise, double* rec,
                    double bussi_c, bool* fused_out) {
    const RunStep r = plan_step(o, k, n_steps, drifted_in, float_precision(ff->precision));
    bool rebuilt = false, fused_ke = false;
    if (drifted_in) {
        int flag = 0;
        MD_CUDA(cudaMemcpyAsync(&flag, nl->flags.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        MD_TRY(sync(s));
        if (flag != 0) MD_TRY(nlist_build(nl, s));
        rebuilt = flag != 0;
    } else {
        MD_TRY(drift_and_update(s, ff, nl, dt, &rebuilt));
    }
    const bool fuse = r.fuse_out && nl->use_tiles && nlist_current(nl, s);
    MD_TRY(forces_list_async(ff, s, nl, want_energy, dt, true, &fused_ke, fuse, drifted_in && !rebuilt));
    *fused_out = fuse;
    MD_TRY(record_energy(ff, s, rec + 3 * k, want_energy));
    bool ke_current = fused_ke;
    if (r.thermo) {
        if (!ke_current) MD_TRY(kinetic_async(s));
        if (r.thermo == 1)
            k_rescale_factor<<<1, 1, 0, s->stream>>>(s->scal.p + kScalKE, dof_of(s->n), r.target, s->scal.p + kScalFactor);
        else
            k_bussi_factor<<<1, 1, 0, s->stream>>>(s->scal.p + kScalKE, dof_of(s->n), o.bussi_temperature, bussi_c,
                                                   noise + k, noise + n_steps + k, s->scal.p + kScalFactor);
        MD_CHECK_LAUNCH();
        MD_TRY(scale_async(s));
        ke_current = false;
    }
    if (r.rdf) MD_TRY(rdf_sample_async(o.rdf, s, nl));
    if (want_ke) {
        if (!ke_current) MD_TRY(ff->precision == MD_PREC_FP64 ? kinetic_async(s) : kinetic_fixed_async(s, ff));
        MD_CUDA(cudaMemcpyAsync(rec + 3 * k + 2, s->scal.p + kScalKE, sizeof(double), cudaMemcpyDeviceToDevice,
                                s->stream));
    }
    return MD_OK;
}

// A chunk whose graph hit an overflow: back to the snapshot, the chunk start's list rebuilt from its reference
// positions (an identity reorder, the same rows; the host grows the capacity or the tile), then the chunk's
// steps on the host path
md_status recover_chunk(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps,
                        const md_run_options& o, int64_t b, int64_t e, bool want_energy, bool want_ke,
                        const double* noise, double* rec, double bussi_c, bool* drifted_io) {
    const size_t N = static_cast<size_t>(s->n);
    cudaStream_t st = s->stream;
    MD_CUDA(s->pos_save.reserve(N));
    MD_CUDA(cudaMemcpyAsync(s->pos_save.p, s->snap_pos.p, sizeof(double4) * N, cudaMemcpyDeviceToDevice, st));
    MD_CUDA(cudaMemcpyAsync(s->pos.p, s->snap_ref.p, sizeof(double4) * N, cudaMemcpyDeviceToDevice, st));
    MD_CUDA(cudaMemcpyAsync(s->vel.p, s->snap_vel.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, st));
    MD_CUDA(cudaMemcpyAsync(s->force.p, s->snap_force.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, st));
    MD_CUDA(cudaMemcpyAsync(s->mass.p, s->snap_mass.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    MD_CUDA(cudaMemcpyAsync(s->ids.p, s->snap_ids.p, sizeof(uint64_t) * N, cudaMemcpyDeviceToDevice, st));
    if (o.rdf && o.rdf->device >= 0)
        MD_CUDA(cudaMemcpyAsync(o.rdf->hist.p, s->snap_hist.p, sizeof(unsigned long long) * o.rdf->bins,
                                cudaMemcpyDeviceToDevice, st));
    const int rebuilds = nl->rebuilds;
    MD_TRY(nlist_build(nl, s));  // positions = the reference positions: the list of the chunk's start
    nl->rebuilds = rebuilds;
    MD_CUDA(cudaMemcpyAsync(s->pos.p, s->pos_save.p, sizeof(double4) * N, cudaMemcpyDeviceToDevice, st));
    MD_CUDA(cudaMemcpyAsync(nl->flags.p, s->snap_flag.p, sizeof(int), cudaMemcpyDeviceToDevice, st));
    // the frames of the chunk's starting positions
    if (nl->use_cells) MD_TRY(frames_async(s, nl));
    if ((ff->precision == MD_PREC_FX64 || ff->precision == MD_PREC_FX32) && nl->use_cells) {
        MD_CUDA(nl->iframes.reserve(N));
        k_frames_fixed<<<blocks_for(static_cast<long long>(N), kThreads), kThreads, 0, st>>>(
            s->pos.p, static_cast<int>(N), nl->cell_sorted.p, nl->grid.ncps, cell_side(nl, s), s->box, nl->iframes.p);
        MD_CHECK_LAUNCH();
    }
    bool drifted = *drifted_io;
    for (int64_t k = b; k < e; ++k)
        MD_TRY(host_step(s, ff, nl, dt, n_steps, o, k, drifted, want_energy, want_ke, noise, rec, bussi_c, &drifted));
    *drifted_io = drifted;
    return MD_OK;
}

// md_run in graph mode (graph_mode_ok holds). A list whose force kernel is not tuned yet runs the first step on
// the host path (the tuning times kernels and waits for them, which a capture cannot); if the host path loses the
// list's tiles (a rebuild found cells too full for them), the run goes on on the host path.
md_status run_steps_graph(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps,
                          const md_run_options& o, double* pe, double* ke, double* virial) {
    const bool want_energy = pe || virial;
    const bool want_ke = ke != nullptr;
    const double bussi_c = o.thermostat == 2 ? std::exp(-dt / o.bussi_tau) : 0.0;
    DevBuf<double> noise, rec;
    if (o.thermostat == 2) {
        MD_CUDA(noise.reserve(2 * static_cast<size_t>(n_steps)));
        MD_CUDA(cudaMemcpyAsync(noise.p, o.bussi_r1, sizeof(double) * n_steps, cudaMemcpyHostToDevice, s->stream));
        MD_CUDA(cudaMemcpyAsync(noise.p + n_steps, o.bussi_chi2, sizeof(double) * n_steps, cudaMemcpyHostToDevice,
                                s->stream));
    }
    MD_CUDA(rec.reserve(3 * static_cast<size_t>(n_steps)));
    bool drifted = false;
    int64_t k0 = 0;
    if (nl->variant[ff->precision] < 0) {
        MD_TRY(host_step(s, ff, nl, dt, n_steps, o, 0, false, want_energy, want_ke, noise.p, rec.p, bussi_c, &drifted));
        k0 = 1;
    }
    const size_t C = static_cast<size_t>(s->graph_chunk);
    bool graphs = graph_mode_ok(s, ff, nl, n_steps);
    if (graphs) {
        MD_TRY(graph_prepare_buffers(s, ff, nl, o));
        MD_TRY(normalize_buffers(s, nl));
    }
    bool rebuilt_on_device = false;
    for (const auto& c : run_chunks(s, k0, n_steps)) {
        const int64_t b = c.first, e = c.second, len = e - b;
        const std::vector<RunStep> steps = chunk_steps(o, b, e, n_steps, float_precision(ff->precision));
        graphs = graphs && graph_mode_ok(s, ff, nl, n_steps) && steps.front().drifted_in == drifted;
        if (!graphs) {  // the host path for the rest of the run
            for (int64_t k = b; k < e; ++k)
                MD_TRY(host_step(s, ff, nl, dt, n_steps, o, k, drifted, want_energy, want_ke, noise.p, rec.p, bussi_c,
                                 &drifted));
            continue;
        }
        RunGraph* g = nullptr;
        MD_TRY(chunk_graph(s, ff, nl, o, steps, dt, want_energy, want_ke, bussi_c, &g));
        if (o.thermostat == 2) {
            MD_CUDA(cudaMemcpyAsync(s->chunk_noise.p, noise.p + b, sizeof(double) * len, cudaMemcpyDeviceToDevice,
                                    s->stream));
            MD_CUDA(cudaMemcpyAsync(s->chunk_noise.p + C, noise.p + n_steps + b, sizeof(double) * len,
                                    cudaMemcpyDeviceToDevice, s->stream));
        }
        // the graph's FP64 energy sums use the records' first buffers: nothing queued may still read them
        MD_TRY(energy_quiesce(ff));
        MD_CUDA(cudaGraphLaunch(g->exec, s->stream));
        MD_CUDA(cudaMemcpyAsync(s->host_scal, s->graph_state.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        MD_TRY(sync(s));
        int state[2];
        std::memcpy(state, s->host_scal, sizeof state);
        s->graph_launches++;
        if (state[1] != 0) {
            s->graph_recoveries++;
            MD_TRY(recover_chunk(s, ff, nl, dt, n_steps, o, b, e, want_energy, want_ke, noise.p, rec.p, bussi_c,
                                 &drifted));
            if (graph_mode_ok(s, ff, nl, n_steps)) MD_TRY(normalize_buffers(s, nl));
            continue;
        }
        drifted = steps.back().fuse_out;
        s->launches += g->kernels + g->body_kernels * static_cast<uint64_t>(state[0]);
        if (state[0] > 0) {  // the rebuilds the graph made, as nlist_build counts them
            rebuilt_on_device = true;
            nl->rebuilds += state[0];
            nl->builds += static_cast<uint64_t>(state[0]);
            if (ff->precision == MD_PREC_FX32) nl->nf_build = nl->builds;
            nl->pairs_ready = false;
            s->layout++;
            nl->layout = s->layout;
        }
        if (g->rdf_samples) {  // src/RadialDistribution.cpp:18-22, per sample
            o.rdf->particles = static_cast<double>(s->n);
            o.rdf->density = o.rdf->particles / std::pow(s->box.L, 3);
            o.rdf->samples += g->rdf_samples;
        }
        if (s->profile) MD_TRY(collect_graph_profile(s, *g));
        MD_CUDA(cudaMemcpyAsync(rec.p + 3 * b, s->chunk_rec.p, sizeof(double) * 3 * len, cudaMemcpyDeviceToDevice,
                                s->stream));
    }
    // the host's record of the tiles (their largest staged count) is stale after rebuilds on the device
    if (rebuilt_on_device) MD_TRY(tile_geometry(nl, s, &nl->use_tiles));
    MD_TRY(join_energy(ff, s));  // records that host steps copied on an energy stream (FP64)
    if (pe || ke || virial) {
        std::vector<double> h(3 * static_cast<size_t>(n_steps));
        MD_CUDA(cudaMemcpyAsync(h.data(), rec.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s->stream));
        MD_TRY(sync(s));
        for (int64_t k = 0; k < n_steps; ++k) {
            if (pe) pe[k] = h[3 * k];
            if (virial) virial[k] = h[3 * k + 1];
            if (ke) ke[k] = h[3 * k + 2];
        }
    }
    if (want_energy) MD_TRY(read_energy(ff, s, nullptr, nullptr, nullptr));
    return sync(s);
}

}  // namespace
