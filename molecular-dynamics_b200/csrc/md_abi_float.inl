// Host orchestration of the float force kernels and of the device-resident step loop (md_run).
// Included by md_abi.cu inside its translation unit.

namespace {

FloatLJ float_lj(const md_forcefield* ff) {
    FloatLJ f{};
    f.sig2 = static_cast<float>(ff->lj.sig2);
    f.eps24 = static_cast<float>(ff->lj.eps24);
    f.eps48 = static_cast<float>(2.0 * ff->lj.eps24);
    f.eps4 = static_cast<float>(ff->lj.eps4);
    f.shift = static_cast<float>(ff->lj.shift);
    f.rc2 = static_cast<float>(ff->lj.rc2);
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

md_status forces_list_float_async(md_forcefield* ff, md_system* s, md_nlist* nl, bool want_energy) {
    const int n = static_cast<int>(s->n);
    const bool fixed = ff->precision == MD_PREC_FP32FX;
    const FloatLJ lj = float_lj(ff);
    MD_CUDA(ff->fx_acc.reserve(4));
    if (want_energy) MD_CUDA(cudaMemsetAsync(ff->fx_acc.p, 0, 3 * sizeof(long long), s->stream));
    auto* acc = reinterpret_cast<unsigned long long*>(ff->fx_acc.p);
    if (n > 0) {
        const unsigned g = blocks_for(n, 128);
        if (nl->use_cells) MD_TRY(frames_async(s, nl));
        const CellOffsets offs = nl->use_cells ? cell_offsets(nl, s) : CellOffsets{};
        // one launch of the float force kernel matching (cells, fixed point, energy)
        auto launch = [&](auto fixed_tag, auto energy_tag) {
            constexpr bool kF = decltype(fixed_tag)::value;
            constexpr bool kE = decltype(energy_tag)::value;
            if (nl->use_cells)
                k_force_fp32<kF, kE><<<g, 128, 0, s->stream>>>(nl->frames.p, n, lj, offs, nl->rows.p, nl->cap,
                                                               nl->counts.p, s->force.p, acc);
            else
                k_force_fp32_small<kF, kE><<<g, 128, 0, s->stream>>>(s->pos.p, n, s->box, lj, nl->rows.p, nl->cap,
                                                                     nl->counts.p, s->force.p, acc);
        };
        using T = std::true_type;
        using F = std::false_type;
        MD_TRY(profile_mark(s));
        if (fixed) {
            if (want_energy) launch(T{}, T{}); else launch(T{}, F{});
        } else {
            if (want_energy) launch(F{}, T{}); else launch(F{}, F{});
        }
        MD_CHECK_LAUNCH();
        MD_TRY(profile_mark(s));
    }
    if (want_energy) {
        k_finish_float_energy<<<1, 1, 0, s->stream>>>(acc, ff->out.p, ff->inside_count.p);
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
    const int n = static_cast<int>(s->n);
    if (n > 0) {
        const size_t smem = sizeof(unsigned int) * r->bins;
        if (smem > 48 * 1024)
            MD_CUDA(cudaFuncSetAttribute(k_rdf_sample, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        k_rdf_sample<<<blocks_for(n, kThreads), kThreads, smem, s->stream>>>(
            s->pos.p, n, s->box, nl->rows.p, nl->cap, nl->counts.p, r->rmax * r->rmax, r->bin_width, r->bins, r->hist.p);
        MD_CHECK_LAUNCH();
    }
    // src/RadialDistribution.cpp:18-22
    const double volume = std::pow(s->box.L, 3);
    r->particles = static_cast<double>(s->n);
    r->density = r->particles / volume;
    r->samples++;
    return MD_OK;
}

// md_run's step loop. This version drives the step from the host and reads the half-skin flag after each
// drift (one 4-byte copy per step), then rebuilds on the host's decision.
md_status run_steps(md_system* s, md_forcefield* ff, md_nlist* nl, double dt, int64_t n_steps,
                    const md_run_options& o, double* pe, double* ke, double* virial) {
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
    for (int64_t k = 0; k < n_steps; ++k) {
        const int64_t step = o.first_step + k;
        const bool current = nlist_current(nl, s);
        MD_TRY(kick_drift_async(s, nl, dt, current));
        bool stale = true;
        if (current) {
            int flag = 0;
            MD_CUDA(cudaMemcpyAsync(&flag, nl->flags.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
            MD_TRY(sync(s));
            stale = flag != 0;
            if (!stale) nl->layout = s->layout;
        }
        if (stale) MD_TRY(nlist_build(nl, s));
        MD_TRY(forces_list_async(ff, s, nl, want_energy));
        MD_TRY(kick_async(s, dt));
        if (want_energy) {
            MD_CUDA(cudaMemcpyAsync(rec.p + 3 * k, ff->out.p, 2 * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
        }
        if (o.thermostat == 1 && o.rescale_every > 0 && step % o.rescale_every == 0) {
            const double target = step <= o.melt_until ? o.melt_temperature : o.rescale_temperature;
            MD_TRY(kinetic_async(s));
            k_rescale_factor<<<1, 1, 0, s->stream>>>(s->scal.p + kScalKE, dof_of(s->n), target, s->scal.p + kScalFactor);
            MD_CHECK_LAUNCH();
            MD_TRY(scale_async(s));
        } else if (o.thermostat == 2) {
            MD_TRY(kinetic_async(s));
            k_bussi_factor<<<1, 1, 0, s->stream>>>(s->scal.p + kScalKE, dof_of(s->n), o.bussi_temperature, bussi_c,
                                                   noise.p + k, noise.p + n_steps + k, s->scal.p + kScalFactor);
            MD_CHECK_LAUNCH();
            MD_TRY(scale_async(s));
        }
        if (o.rdf && o.rdf_every > 0 && step % o.rdf_every == 0) MD_TRY(rdf_sample_async(o.rdf, s, nl));
        if (ke) {
            MD_TRY(kinetic_async(s));
            MD_CUDA(cudaMemcpyAsync(rec.p + 3 * k + 2, s->scal.p + kScalKE, sizeof(double), cudaMemcpyDeviceToDevice,
                                    s->stream));
        }
    }
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
