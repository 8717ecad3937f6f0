// Host orchestration of the float force kernels and of the device-resident step loop (md_run).
// Included by md_abi.cu inside its translation unit.

namespace {

// md_run's graph mode (md_run_graph.inl)
bool graph_mode_ok(const md_system* s, const md_forcefield* ff, const md_nlist* nl, int64_t n_steps);
md_status run_steps_graph(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps,
                          const md_run_options& o, double* pe, double* ke, double* virial);

FloatLJ float_lj(const md_forcefield* ff) {
    FloatLJ f{};
    f.sig2 = static_cast<float>(ff->lj.sig2);
    f.eps24 = static_cast<float>(ff->lj.eps24);
    f.eps48 = static_cast<float>(2.0 * ff->lj.eps24);
    f.eps4 = static_cast<float>(ff->lj.eps4);
    f.shift = static_cast<float>(ff->lj.shift);
    f.rc2 = static_cast<float>(ff->lj.rc2);
    // the float r^2 of a pair is within ~1e-5 of the exact value (frames are cell-relative), so this shell
    // holds every pair whose float and double cutoff tests could disagree
    f.band = static_cast<float>(1e-5 * ff->lj.rc2 + 1e-4);
    f.rc2d = ff->lj.rc2;
    return f;
}

double cell_side(const md_nlist* nl, const md_system* s) { return s->box.L / nl->grid.ncps; }

CellOffsets cell_offsets(const md_nlist* nl, const md_system* s) {
    CellOffsets o{};
    const double cs = cell_side(nl, s);
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                const int code = (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
                o.off[code] = make_float4(static_cast<float>(-dx * cs), static_cast<float>(-dy * cs),
                                          static_cast<float>(-dz * cs), 0.0f);
            }
    return o;
}

md_status frames_async(md_system* s, md_nlist* nl) {
    const int n = static_cast<int>(s->n);
    MD_CUDA(nl->frames.reserve(static_cast<size_t>(n) + 1));
    k_frames<<<blocks_for(n + 1, kThreads), kThreads, 0, s->stream>>>(s->pos.p, n, nl->cell_sorted.p, nl->grid.ncps,
                                                                      cell_side(nl, s), s->box, nl->frames.p);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

Fx64LJ fx64_lj(const md_forcefield* ff) {
    Fx64LJ f{};
    f.lj = ff->lj;
    f.eps48 = 2.0 * ff->lj.eps24;
    // the fixed-point separation is exact to ~4e-9, so r^2 is within ~3e-8 of the reference's
    f.band = 1e-6 * ff->lj.rc2;
    return f;
}

FixedOffsets fixed_offsets(const md_nlist* nl, const md_system* s) {
    FixedOffsets o{};
    const int cellq = static_cast<int>(std::llrint(cell_side(nl, s) * kFrameScale));
    for (int code = 0; code < 27; ++code) {
        const int d[3] = {code / 9 - 1, (code / 3) % 3 - 1, code % 3 - 1};
        o.off[code] = make_int4(-d[0] * cellq, -d[1] * cellq, -d[2] * cellq, 0);
    }
    return o;
}

// MD_PREC_FX64 list forces: fixed-point frames of the current positions, then the global-gather kernel (or the
// small-box kernel under 3 cells per side); the closing kick and kinetic energy are fused as in the float modes
// fixed_fresh: the fixed-point frames already match the positions (the previous force kernel drifted them and
// there was no rebuild since); fuse_drift: as in forces_list_float_async, writing fixed-point frames
md_status forces_list_fx64_async(md_forcefield* ff, md_system* s, md_nlist* nl, bool want_energy, double kick_dt,
                                 bool* fused_ke, bool fixed_fresh, bool fuse_drift) {
    const int n = static_cast<int>(s->n);
    const bool kick = kick_dt > 0.0;
    const Fx64LJ lj = fx64_lj(ff);
    MD_CUDA(ff->fx_acc.reserve(4));
    if (want_energy || kick) MD_CUDA(cudaMemsetAsync(ff->fx_acc.p, 0, 4 * sizeof(long long), s->stream));
    auto* acc = reinterpret_cast<unsigned long long*>(ff->fx_acc.p);
    nl->variant[MD_PREC_FX64] = 0;
    if (n > 0) {
        const unsigned g = blocks_for(n, 128);
        KickArgs ka{kick ? s->vel.p : nullptr, s->mass.p, 0.5 * kick_dt};
        if (nl->use_cells) {
            MD_CUDA(nl->iframes.reserve(n));
            if (!fixed_fresh) {
                k_frames_fixed<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(s->pos.p, n, nl->cell_sorted.p,
                                                                                   nl->grid.ncps, cell_side(nl, s),
                                                                                   s->box, nl->iframes.p);
                MD_CHECK_LAUNCH();
            }
            const bool fuse = fuse_drift && kick;
            if (fuse) {  // the next step's kick and drift, new positions and fixed-point frames to spare buffers
                MD_CUDA(s->pos2.reserve(n));
                MD_CUDA(nl->iframes2.reserve(n));
                MD_CUDA(cudaMemsetAsync(nl->flags.p, 0, sizeof(int), s->stream));
                ka.pos_in = s->pos.p;
                ka.pos_out = s->pos2.p;
                ka.iframes_out = nl->iframes2.p;
                ka.ref_pos = nl->ref_pos.p;
                ka.max_disp2 = nl->max_disp2;
                ka.stale = nl->flags.p;
                ka.cell_sorted = nl->cell_sorted.p;
                ka.ncps = nl->grid.ncps;
                ka.cell = cell_side(nl, s);
                ka.dt = kick_dt;
                ka.box = s->box;
            }
            const FixedOffsets offs = fixed_offsets(nl, s);
            MD_TRY(profile_mark(s));
            if (want_energy)
                k_force_fx64_rows<true><<<g, 128, 0, s->stream>>>(nl->iframes.p, s->pos.p, n, s->box, lj, offs, nl->rows.p,
                                                                  nl->cap, nl->counts.p, s->force.p, acc, ka);
            else
                k_force_fx64_rows<false><<<g, 128, 0, s->stream>>>(nl->iframes.p, s->pos.p, n, s->box, lj, offs,
                                                                   nl->rows.p, nl->cap, nl->counts.p, s->force.p, acc, ka);
            if (fuse) {
                MD_CHECK_LAUNCH();
                swap_buffers(s->pos, s->pos2);
                swap_buffers(nl->iframes, nl->iframes2);
            }
        } else {
            MD_TRY(profile_mark(s));
            if (want_energy)
                k_force_fx64_small<true><<<g, 128, 0, s->stream>>>(s->pos.p, n, s->box, lj, nl->rows.p, nl->cap,
                                                                   nl->counts.p, s->force.p, acc, ka);
            else
                k_force_fx64_small<false><<<g, 128, 0, s->stream>>>(s->pos.p, n, s->box, lj, nl->rows.p, nl->cap,
                                                                    nl->counts.p, s->force.p, acc, ka);
        }
        MD_CHECK_LAUNCH();
        MD_TRY(profile_mark(s));
    }
    const bool ke_fused = kick && n > 0;
    if (want_energy || ke_fused) {
        k_finish_float_energy<<<1, 1, 0, s->stream>>>(acc, ff->out.p, ff->inside_count.p,
                                                      ke_fused ? s->scal.p + kScalKE : nullptr, 1.0 / kKineticScale,
                                                      kEnergyUnit64);
        MD_CHECK_LAUNCH();
    }
    if (fused_ke) *fused_ke = ke_fused;
    return MD_OK;
}

// MD_PREC_FX32 evaluates pairs closer than this many sigma (plus the skin, at the list build) in double
constexpr double kFx32NearSigma = 1.2;

// MD_PREC_FX32's near and far rows of the rows just built, classified on ref_frames (the float frames of the
// build's positions): k_rows_split, then k_rows_split_fix for the rows with more near entries than a near row
// holds. rows_nf holds the near rows and, after them, the far rows.
md_status split_rows_async(md_system* s, md_nlist* nl, const float4* ref_frames, float near2, cudaStream_t st) {
    const int n = static_cast<int>(s->n);
    uint32_t* near_rows = nl->rows_nf.p;
    uint32_t* far_rows = nl->rows_nf.p + fx32_near_entries(n);
    k_rows_split<<<blocks_for(n, kSplitThreads), kSplitThreads, 0, st>>>(
        ref_frames, n, cell_offsets(nl, s), near2, nl->rows.p, nl->cap, nl->counts.p, near_rows, far_rows,
        nl->counts_nf.p);
    MD_CHECK_LAUNCH();
    k_rows_split_fix<<<std::min(blocks_for(n, 128), 1184u), 128, 0, st>>>(ref_frames, n, cell_offsets(nl, s), near2,
                                                                         nl->rows.p, nl->cap, nl->counts.p, near_rows,
                                                                         far_rows, nl->counts_nf.p);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

// MD_PREC_FX32's near and far rows of the list's last build, made once per build and near radius. The
// classification reads the float frames of the list's reference positions, made here into the spare frame buffer
// (free between steps; a fused force kernel writes it only after this).
md_status ensure_near_first(md_forcefield* ff, md_system* s, md_nlist* nl) {
    const int n = static_cast<int>(s->n);
    const double near = kFx32NearSigma * ff->sigma + nl->skin;
    const double near2 = near * near;
    if (n == 0 || (nl->nf_build == nl->builds && nl->nf_near2 == near2)) return MD_OK;
    const size_t entries = fx32_near_entries(n) + row_buffer_entries(n, nl->cap);
    if (entries / 4 > 0xffffffffull) return fail(MD_ERR_INVALID, "MD_PREC_FX32: the split rows exceed 2^32 quads");
    MD_CUDA(nl->rows_nf.reserve(entries));
    MD_CUDA(nl->counts_nf.reserve(n));
    MD_CUDA(nl->frames2.reserve(static_cast<size_t>(n) + 1));
    k_frames<<<blocks_for(n + 1, kThreads), kThreads, 0, s->stream>>>(nl->ref_pos.p, n, nl->cell_sorted.p,
                                                                      nl->grid.ncps, cell_side(nl, s), s->box,
                                                                      nl->frames2.p);
    MD_CHECK_LAUNCH();
    MD_TRY(split_rows_async(s, nl, nl->frames2.p, static_cast<float>(near2), s->stream));
    nl->nf_build = nl->builds;
    nl->nf_near2 = near2;
    return MD_OK;
}

// MD_PREC_FX32 list forces: after each list build the rows are split into near and far rows (once per
// build and near radius); then the fixed-point frames and k_force_fx32 on a resident grid, with the closing kick,
// kinetic energy and optionally the next drift fused as in forces_list_fx64_async. Boxes under 3 cells per side
// take the MD_PREC_FX64 small-box kernel (every pair in double).
md_status forces_list_fx32_async(md_forcefield* ff, md_system* s, md_nlist* nl, bool want_energy, double kick_dt,
                                 bool* fused_ke, bool frames_fresh, bool fixed_fresh, bool fuse_drift) {
    if (!nl->use_cells) return forces_list_fx64_async(ff, s, nl, want_energy, kick_dt, fused_ke, fixed_fresh, fuse_drift);
    const int n = static_cast<int>(s->n);
    const bool kick = kick_dt > 0.0;
    const Fx64LJ dlj = fx64_lj(ff);
    const FloatLJ flj = float_lj(ff);
    MD_CUDA(ff->fx_acc.reserve(4));
    if (want_energy || kick) MD_CUDA(cudaMemsetAsync(ff->fx_acc.p, 0, 4 * sizeof(long long), s->stream));
    auto* acc = reinterpret_cast<unsigned long long*>(ff->fx_acc.p);
    nl->variant[MD_PREC_FX32] = 0;
    if (n > 0) {
        MD_TRY(ensure_near_first(ff, s, nl));
        if (!frames_fresh) MD_TRY(frames_async(s, nl));
        MD_CUDA(nl->iframes.reserve(n));
        if (!fixed_fresh) {
            k_frames_fixed<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(s->pos.p, n, nl->cell_sorted.p,
                                                                               nl->grid.ncps, cell_side(nl, s), s->box,
                                                                               nl->iframes.p);
            MD_CHECK_LAUNCH();
        }
        KickArgs ka{kick ? s->vel.p : nullptr, s->mass.p, 0.5 * kick_dt};
        const bool fuse = fuse_drift && kick;
        if (fuse) {  // the next step's kick and drift, new positions and both kinds of frames to spare buffers
            MD_CUDA(s->pos2.reserve(n));
            MD_CUDA(nl->iframes2.reserve(n));
            MD_CUDA(nl->frames2.reserve(static_cast<size_t>(n) + 1));
            MD_CUDA(cudaMemsetAsync(nl->flags.p, 0, sizeof(int), s->stream));
            ka.pos_in = s->pos.p;
            ka.pos_out = s->pos2.p;
            ka.iframes_out = nl->iframes2.p;
            ka.frames_out = nl->frames2.p;
            ka.ref_pos = nl->ref_pos.p;
            ka.max_disp2 = nl->max_disp2;
            ka.stale = nl->flags.p;
            ka.cell_sorted = nl->cell_sorted.p;
            ka.ncps = nl->grid.ncps;
            ka.cell = cell_side(nl, s);
            ka.dt = kick_dt;
            ka.box = s->box;
        }
        const FixedOffsets offs = fixed_offsets(nl, s);
        const CellOffsets foffs = cell_offsets(nl, s);
        auto go = [&](auto kernel, unsigned& grid) -> md_status {
            if (grid == 0) {
                int sms = 0, per_sm = 0;
                MD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
                MD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0));
                grid = static_cast<unsigned>(std::max(1, sms * per_sm));
            }
            MD_TRY(profile_mark(s));
            kernel<<<std::min(blocks_for(n, 128), grid), 128, 0, s->stream>>>(
                nl->iframes.p, nl->frames.p, s->pos.p, n, s->box, dlj, flj, offs, foffs,
                reinterpret_cast<const uint4*>(nl->rows_nf.p), static_cast<unsigned>(fx32_near_entries(n) / 4), nl->cap,
                nl->counts_nf.p, s->force.p, acc, ka);
            MD_CHECK_LAUNCH();
            return profile_mark(s);
        };
        if (want_energy)
            MD_TRY(go(k_force_fx32<true>, s->fx32_resident[1]));
        else
            MD_TRY(go(k_force_fx32<false>, s->fx32_resident[0]));
        if (fuse) {
            swap_buffers(s->pos, s->pos2);
            swap_buffers(nl->iframes, nl->iframes2);
            swap_buffers(nl->frames, nl->frames2);
        }
    }
    const bool ke_fused = kick && n > 0;
    if (want_energy || ke_fused) {
        k_finish_float_energy<<<1, 1, 0, s->stream>>>(acc, ff->out.p, ff->inside_count.p,
                                                      ke_fused ? s->scal.p + kScalKE : nullptr, 1.0 / kKineticScale,
                                                      kEnergyUnit64);
        MD_CHECK_LAUNCH();
    }
    if (fused_ke) *fused_ke = ke_fused;
    return MD_OK;
}

// See forces_list_async. Every float kernel fuses the closing kick with a fixed-point kinetic energy.
md_status forces_list_float_async(md_forcefield* ff, md_system* s, md_nlist* nl, bool want_energy, double kick_dt,
                                  bool frames_fresh, bool* fused_ke, bool fuse_drift, bool fixed_fresh) {
    if (ff->precision == MD_PREC_FX64)
        return forces_list_fx64_async(ff, s, nl, want_energy, kick_dt, fused_ke, fixed_fresh, fuse_drift);
    if (ff->precision == MD_PREC_FX32)
        return forces_list_fx32_async(ff, s, nl, want_energy, kick_dt, fused_ke, frames_fresh, fixed_fresh, fuse_drift);
    const int n = static_cast<int>(s->n);
    const bool fixed = ff->precision == MD_PREC_FP32FX;
    const bool kick = kick_dt > 0.0;
    const FloatLJ lj = float_lj(ff);
    MD_CUDA(ff->fx_acc.reserve(4));
    if (want_energy || kick) MD_CUDA(cudaMemsetAsync(ff->fx_acc.p, 0, 4 * sizeof(long long), s->stream));
    auto* acc = reinterpret_cast<unsigned long long*>(ff->fx_acc.p);
    if (n > 0) {
        const unsigned g = blocks_for(n, 128);
        if (nl->use_cells) {
            // variant 0: global gathers (k_force_fp32_rows); 1: shared-memory tile; 2: global gathers with the rows
            // prefetched a group ahead; 3: as 2 with capped registers; 4: as 2 on a resident grid with split offset
            // tables (all the same bits)
            if (!frames_fresh) MD_TRY(frames_async(s, nl));
            const TileGeom& tg = nl->tiles_geom;
            const CellOffsets offs = cell_offsets(nl, s);
            const size_t smem = sizeof(float4) * (tg.max_staged + 1);
            KickArgs drift{nullptr, nullptr, 0.0};
            auto launch = [&](int variant, bool with_kick, bool energy, double* tune_vel = nullptr,
                              const KickArgs* fused = nullptr) -> md_status {
                KickArgs ka = fused ? *fused
                                    : tune_vel ? KickArgs{tune_vel, s->mass.p, 0.0}
                                               : KickArgs{with_kick ? s->vel.p : nullptr, s->mass.p, 0.5 * kick_dt};
                ka.overflow = g_graph_overflow;
                auto go = [&](auto rows_kernel, auto tile_kernel, auto prefetch_kernel, auto capped_kernel,
                              auto resident_kernel) -> md_status {
                    if (variant == 4) {
                        unsigned& grid = s->fp32_resident[fixed ? 1 : 0][energy ? 1 : 0];
                        if (grid == 0) {
                            int sms = 0, per_sm = 0;
                            MD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
                            MD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, resident_kernel, 128, 0));
                            grid = static_cast<unsigned>(std::max(1, sms * per_sm));
                        }
                        resident_kernel<<<std::min(g, grid), 128, 0, s->stream>>>(
                            nl->frames.p, s->pos.p, n, s->box, lj, offs, nl->rows.p, nl->cap, nl->counts.p, s->force.p,
                            acc, ka);
                    } else if (variant == 1) {
                        MD_CUDA(allow_smem(tile_kernel, smem));
                        tile_kernel<<<tile_blocks(tg), kTileThreads, smem, s->stream>>>(
                            nl->frames.p, s->pos.p, n, nl->grid.start.p, nl->cell_sorted.p, tg, lj, offs, nl->rows.p,
                            nl->cap, nl->counts.p, s->force.p, acc, ka);
                    } else if (variant == 2) {
                        prefetch_kernel<<<g, 128, 0, s->stream>>>(nl->frames.p, s->pos.p, n, s->box, lj, offs,
                                                                  nl->rows.p, nl->cap, nl->counts.p, s->force.p, acc, ka);
                    } else if (variant == 3) {
                        capped_kernel<<<g, 128, 0, s->stream>>>(nl->frames.p, s->pos.p, n, s->box, lj, offs, nl->rows.p,
                                                                nl->cap, nl->counts.p, s->force.p, acc, ka);
                    } else {
                        rows_kernel<<<g, 128, 0, s->stream>>>(nl->frames.p, s->pos.p, n, s->box, lj, offs, nl->rows.p,
                                                              nl->cap, nl->counts.p, s->force.p, acc, ka);
                    }
                    MD_CHECK_LAUNCH();
                    return MD_OK;
                };
                if (fixed)
                    return energy ? go(k_force_fp32_rows<true, true>, k_force_fp32_tile<true, true>,
                                       k_force_fp32_rows<true, true, true>, k_force_fp32_rows<true, true, true, 7>,
                                       k_force_fp32_resident<true, true>)
                                  : go(k_force_fp32_rows<true, false>, k_force_fp32_tile<true, false>,
                                       k_force_fp32_rows<true, false, true>, k_force_fp32_rows<true, false, true, 7>,
                                       k_force_fp32_resident<true, false>);
                return energy ? go(k_force_fp32_rows<false, true>, k_force_fp32_tile<false, true>,
                                   k_force_fp32_rows<false, true, true>, k_force_fp32_rows<false, true, true, 7>,
                                   k_force_fp32_resident<false, true>)
                              : go(k_force_fp32_rows<false, false>, k_force_fp32_tile<false, false>,
                                   k_force_fp32_rows<false, false, true>, k_force_fp32_rows<false, false, true, 7>,
                                   k_force_fp32_resident<false, false>);
            };
            // tune on the kernel the steps run (energy and the fused kick), the kick writing into the reorder
            // buffer (3n doubles, idle between rebuilds) so the state is untouched
            MD_CUDA(s->vel2.reserve(3 * static_cast<size_t>(n)));
            MD_TRY(choose_variant(s, nl, ff->precision, [&](int v) { return launch(v, true, true, s->vel2.p); }));
            if (want_energy || kick) MD_CUDA(cudaMemsetAsync(ff->fx_acc.p, 0, 4 * sizeof(long long), s->stream));
            MD_TRY(profile_mark(s));
            if (fuse_drift && kick && nl->use_tiles) {
                // the next step's kick and drift in the same kernel: new positions and frames go to the spare
                // buffers (the force loop reads the current ones) and are swapped in after the launch
                MD_CUDA(s->pos2.reserve(n));
                MD_CUDA(nl->frames2.reserve(static_cast<size_t>(n) + 1));
                MD_CUDA(cudaMemsetAsync(nl->flags.p, 0, sizeof(int), s->stream));
                drift = KickArgs{s->vel.p, s->mass.p, 0.5 * kick_dt};
                drift.pos_in = s->pos.p;
                drift.pos_out = s->pos2.p;
                drift.frames_out = nl->frames2.p;
                drift.ref_pos = nl->ref_pos.p;
                drift.max_disp2 = nl->max_disp2;
                drift.stale = nl->flags.p;
                drift.cell_sorted = nl->cell_sorted.p;
                drift.ncps = tg.ncps;
                drift.cell = tg.cell;
                drift.dt = kick_dt;
                drift.box = s->box;
                MD_TRY(launch(nl->variant[ff->precision], kick, want_energy, nullptr, &drift));
                swap_buffers(s->pos, s->pos2);
                swap_buffers(nl->frames, nl->frames2);
            } else {
                MD_TRY(launch(nl->variant[ff->precision], kick, want_energy));
            }
            MD_TRY(profile_mark(s));
        } else {
            const KickArgs ka{kick ? s->vel.p : nullptr, s->mass.p, 0.5 * kick_dt};
            MD_TRY(profile_mark(s));
            if (fixed) {
                if (want_energy)
                    k_force_fp32_small<true, true><<<g, 128, 0, s->stream>>>(s->pos.p, n, s->box, lj, nl->rows.p,
                                                                             nl->cap, nl->counts.p, s->force.p, acc, ka);
                else
                    k_force_fp32_small<true, false><<<g, 128, 0, s->stream>>>(s->pos.p, n, s->box, lj, nl->rows.p,
                                                                              nl->cap, nl->counts.p, s->force.p, acc, ka);
            } else {
                if (want_energy)
                    k_force_fp32_small<false, true><<<g, 128, 0, s->stream>>>(s->pos.p, n, s->box, lj, nl->rows.p,
                                                                              nl->cap, nl->counts.p, s->force.p, acc, ka);
                else
                    k_force_fp32_small<false, false><<<g, 128, 0, s->stream>>>(s->pos.p, n, s->box, lj, nl->rows.p,
                                                                               nl->cap, nl->counts.p, s->force.p, acc, ka);
            }
            MD_CHECK_LAUNCH();
            MD_TRY(profile_mark(s));
        }
    }
    const bool ke_fused = kick && n > 0;
    if (want_energy || ke_fused) {
        k_finish_float_energy<<<1, 1, 0, s->stream>>>(acc, ff->out.p, ff->inside_count.p,
                                                      ke_fused ? s->scal.p + kScalKE : nullptr, 1.0 / kKineticScale);
        MD_CHECK_LAUNCH();
    }
    if (fused_ke) *fused_ke = ke_fused;
    return MD_OK;
}

// Fixed-point kinetic energy of the current velocities into s->scal[kScalKE] (float runs)
md_status kinetic_fixed_async(md_system* s, md_forcefield* ff) {
    const int n = static_cast<int>(s->n);
    MD_CUDA(ff->fx_acc.reserve(4));
    auto* acc = reinterpret_cast<unsigned long long*>(ff->fx_acc.p) + 3;
    MD_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long), s->stream));
    if (n > 0) {
        k_kinetic_fixed<<<blocks_for(n, kThreads), kThreads, 0, s->stream>>>(s->vel.p, s->mass.p, n, acc);
        MD_CHECK_LAUNCH();
    }
    k_fixed_to_double<<<1, 1, 0, s->stream>>>(acc, 1.0 / kKineticScale, s->scal.p + kScalKE);
    MD_CHECK_LAUNCH();
    return MD_OK;
}

// The histogram kernel of RadialDistribution::sample (src/RadialDistribution.cpp:11-30) on the system's stream; the
// histogram must exist
md_status rdf_kernel_async(md_rdf* r, md_system* s, md_nlist* nl) {
    const int n = static_cast<int>(s->n);
    if (n > 0) {
        const size_t smem = sizeof(unsigned int) * r->bins;
        MD_CUDA(allow_smem(k_rdf_sample, smem));
        k_rdf_sample<<<blocks_for(n, kThreads), kThreads, smem, s->stream>>>(
            s->pos.p, n, s->box, nl->rows.p, nl->cap, nl->counts.p, r->rmax * r->rmax, r->bin_width, r->bins, r->hist.p);
        MD_CHECK_LAUNCH();
    }
    return MD_OK;
}

// RadialDistribution::sample (src/RadialDistribution.cpp:11-30) queued on the system's stream
md_status rdf_sample_async(md_rdf* r, md_system* s, md_nlist* nl) {
    if (r->device < 0) {
        r->device = s->device;
        MD_CUDA(r->hist.reserve(r->bins));
        MD_CUDA(cudaMemsetAsync(r->hist.p, 0, sizeof(unsigned long long) * r->bins, s->stream));
    }
    MD_TRY(rdf_kernel_async(r, s, nl));
    // src/RadialDistribution.cpp:18-22
    const double volume = std::pow(s->box.L, 3);
    r->particles = static_cast<double>(s->n);
    r->density = r->particles / volume;
    r->samples++;
    return MD_OK;
}

// The force-kernel times of one chunk graph's launch (md_profile_*): the stream must have been synchronised
md_status collect_graph_profile(md_system* s, const RunGraph& g) {
    for (size_t k = 0; k + 1 < g.prof.size(); k += 2) {
        float ms = 0.f;
        MD_CUDA(cudaEventElapsedTime(&ms, g.prof[k], g.prof[k + 1]));
        s->profile_ms += ms;
        s->profile_count++;
    }
    return MD_OK;
}

// md_run's step loop. The step is driven from the host, which reads the half-skin flag after each drift (one
// 4-byte copy per step) and rebuilds on its decision. Kinetic energies: FP64 runs use the reference's blocked
// summation order (so thermostats stay bit-identical); float runs use the fixed-point kinetic energy the force
// kernel fuses with the closing kick, and recompute it after a thermostat.
md_status run_steps(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps,
                    const md_run_options& o, double* pe, double* ke, double* virial) {
    // graphs when the run amortises their capture (two chunks or more) or md_run_prepare captured them for it
    if (graph_mode_ok(s, ff, nl, n_steps) && (n_steps >= 2 * static_cast<int64_t>(s->graph_chunk) ||
                                              n_steps == s->prepared_steps))
        return run_steps_graph(s, ff, nl, dt, n_steps, o, pe, ke, virial);
    const double bussi_c = o.thermostat == 2 ? std::exp(-dt / o.bussi_tau) : 0.0;  // src/Thermostat.cpp:46
    DevBuf<double> noise;
    if (o.thermostat == 2 && n_steps > 0) {
        MD_CUDA(noise.reserve(2 * static_cast<size_t>(n_steps)));
        MD_CUDA(cudaMemcpyAsync(noise.p, o.bussi_r1, sizeof(double) * n_steps, cudaMemcpyHostToDevice, s->stream));
        MD_CUDA(cudaMemcpyAsync(noise.p + n_steps, o.bussi_chi2, sizeof(double) * n_steps, cudaMemcpyHostToDevice,
                                s->stream));
    }
    DevBuf<double> rec;  // per step: pe, virial, ke
    if (n_steps > 0) MD_CUDA(rec.reserve(3 * static_cast<size_t>(n_steps)));
    const bool want_energy = pe || virial;
    const bool exact_ke = ff->precision == MD_PREC_FP64;
    const bool float_mode = ff->precision == MD_PREC_FP32FX || ff->precision == MD_PREC_FP32 ||
                            ff->precision == MD_PREC_FX64 || ff->precision == MD_PREC_FX32;
    bool drifted = false;  // the previous step's force kernel already made this step's kick and drift
    for (int64_t k = 0; k < n_steps; ++k) {
        const int64_t step = o.first_step + k;
        bool rebuilt = false, fused_ke = false;
        if (drifted) {
            int flag = 0;
            MD_CUDA(cudaMemcpyAsync(&flag, nl->flags.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
            MD_TRY(sync(s));
            if (flag != 0) MD_TRY(nlist_build(nl, s));
            rebuilt = flag != 0;
        } else {
            MD_TRY(drift_and_update(s, ff, nl, dt, &rebuilt));
        }
        // fuse the next step's kick and drift unless something touches velocities or positions in between
        const bool thermostat_now = (o.thermostat == 1 && o.rescale_every > 0 && step % o.rescale_every == 0) ||
                                    o.thermostat == 2;
        const bool rdf_now = o.rdf && o.rdf_every > 0 && step % o.rdf_every == 0;
        const bool fuse = float_mode && k + 1 < n_steps && !thermostat_now && !rdf_now && nl->use_tiles &&
                          nlist_current(nl, s);
        // FX64's fixed-point frames are current when the previous force kernel wrote them and nothing rebuilt
        const bool fixed_fresh = drifted && !rebuilt;
        MD_TRY(forces_list_async(ff, s, nl, want_energy, dt, true, &fused_ke, fuse, fixed_fresh));
        drifted = fuse;
        if (want_energy) {  // on the stream where this step's sums end (FP64: the force field's chain stream)
            const cudaStream_t es = energy_stream(ff, s);
            MD_CUDA(cudaMemcpyAsync(rec.p + 3 * k, ff->out.p, 2 * sizeof(double), cudaMemcpyDeviceToDevice, es));
            if (es != s->stream) MD_CUDA(cudaEventRecord(ff->ev_done, es));  // the join covers the copy too
        }
        bool ke_current = fused_ke && !exact_ke;  // scal[kScalKE] holds this step's kinetic energy
        const bool rescale = o.thermostat == 1 && o.rescale_every > 0 && step % o.rescale_every == 0;
        if (rescale || o.thermostat == 2) {
            if (!ke_current) MD_TRY(kinetic_async(s));
            if (rescale) {
                const double target = step <= o.melt_until ? o.melt_temperature : o.rescale_temperature;
                k_rescale_factor<<<1, 1, 0, s->stream>>>(s->scal.p + kScalKE, dof_of(s->n), target,
                                                         s->scal.p + kScalFactor);
            } else {
                k_bussi_factor<<<1, 1, 0, s->stream>>>(s->scal.p + kScalKE, dof_of(s->n), o.bussi_temperature, bussi_c,
                                                       noise.p + k, noise.p + n_steps + k, s->scal.p + kScalFactor);
            }
            MD_CHECK_LAUNCH();
            MD_TRY(scale_async(s));
            ke_current = false;
        }
        if (o.rdf && o.rdf_every > 0 && step % o.rdf_every == 0) MD_TRY(rdf_sample_async(o.rdf, s, nl));
        if (ke) {
            if (!ke_current) MD_TRY(exact_ke ? kinetic_async(s) : kinetic_fixed_async(s, ff));
            MD_CUDA(cudaMemcpyAsync(rec.p + 3 * k + 2, s->scal.p + kScalKE, sizeof(double), cudaMemcpyDeviceToDevice,
                                    s->stream));
        }
    }
    MD_TRY(join_energy(ff, s));
    if (n_steps > 0 && (pe || ke || virial)) {
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
