// batch_host.inl -- swd_rtm_batch: many shots of uneven record length and receiver aperture
// through batched launches (part of swd.cu's translation unit).
//
// A batch of B shots runs as one launch per half step with blockIdx.z = shot.  Every
// per-shot grid array (wavefields, dp/dt, FP64 images) is one allocation of B slices with a
// fixed stride, so a kernel reaches its shot's slice by one offset; per-shot scalars (source
// cell, nt, trace / wavelet / well-map offsets) come from a small descriptor table.  Shots
// are sorted by record length so a batch's records end close together; in the forward pass
// a shot whose record has ended returns at once, and in the backward pass each shot runs
// from its own nt - 2 down to 0 (it = counter + tshift).  Both time loops are chunked CUDA
// graphs whose arguments do not change from batch to batch, so they are captured once.  The
// batch size is chosen by timing short probes of B = 1, 2, 4, 8 on the first batch (the
// autotuner) unless fixed with swd_set_option(SWD_OPT_BATCH).

template <int LC>
static void launch_fwd_batch(const FwdArgs &a, dim3 grid, cudaStream_t s, cudaEvent_t *ev)
{
    if (ev) cudaEventRecordWithFlags(ev[0], s, cudaEventRecordExternal);
    k_fwd_v<LC, 1, false, true><<<grid, dim3(32, 8), 0, s>>>(a);
    if (ev) { cudaEventRecordWithFlags(ev[1], s, cudaEventRecordExternal); cudaEventRecordWithFlags(ev[2], s, cudaEventRecordExternal); }
    k_fwd_p<LC, 1, FP_PLAIN, true><<<grid, dim3(32, 8), 0, s>>>(a);
    if (ev) cudaEventRecordWithFlags(ev[3], s, cudaEventRecordExternal);
}

template <int LC>
static void launch_bwd_batch(const BwdArgs &a, dim3 grid, cudaStream_t s, cudaEvent_t *ev, int by_kind)
{
    if (ev) cudaEventRecordWithFlags(ev[0], s, cudaEventRecordExternal);
    if (by_kind) k_bwd_v<LC, true><<<grid, dim3(32, 8), 0, s>>>(a);
    else k_bwd_1<LC, true><<<grid, dim3(32, 8), 0, s>>>(a);
    if (ev) { cudaEventRecordWithFlags(ev[1], s, cudaEventRecordExternal); cudaEventRecordWithFlags(ev[2], s, cudaEventRecordExternal); }
    if (by_kind) k_bwd_p<LC, true><<<grid, dim3(32, 8), 0, s>>>(a);
    else k_bwd_2<LC, true><<<grid, dim3(32, 8), 0, s>>>(a);
    if (ev) cudaEventRecordWithFlags(ev[3], s, cudaEventRecordExternal);
}

// elements between consecutive shots' slices of a batched grid array (guards included)
static size_t batch_stride(const swd_ctx *c) { return (size_t)c->ntx * c->ldz + 2 * GUARD; }

// nb zeroed slices; element 0 of slice 0 sits after its guard band
static int ensure_bgrid(swd_ctx *ctx, DevBuf &b, size_t elem, int nb)
{
    const size_t n = batch_stride(ctx) * nb * elem;
    CKR(ensure(ctx, b, n));
    b.off = GUARD * elem;
    CK(cudaMemsetAsync(b.p, 0, n, ctx->stream));
    return SWD_OK;
}

static Wave batch_wave(swd_ctx *c, int k)
{
    Wave w;
    w.p = F(c->bat.w[k][0]); w.vx = F(c->bat.w[k][1]); w.vz = F(c->bat.w[k][2]);
    w.ppx = F(c->bat.w[k][3]); w.ppz = F(c->bat.w[k][4]); w.pvx = F(c->bat.w[k][5]); w.pvz = F(c->bat.w[k][6]);
    return w;
}

// One batch: shots[idx[0..nb)].  probe_steps > 0 runs only that many forward and backward
// steps and skips the per-shot post (autotuner probes; the stack is left alone).
static int rtm_batch_run(swd_ctx *ctx, const swd_shot *shots, const float *const *ricks, const float *const *data,
                         const int *idx, int nb, unsigned flags, int probe_steps)
{
    std::vector<ShotPlan> P(nb);
    std::vector<ShotDesc> desc(nb);
    int ntmax = 0, wells = 0, wav_total = 0;
    long long seis_total = 0;
    for (int b = 0; b < nb; b++) {
        const swd_shot *s = &shots[idx[b]];
        CKR(plan_shot_host(ctx, s, P[b]));
        ntmax = std::max(ntmax, s->nt);
        ShotDesc &d = desc[b];
        d.sx = s->s_ix; d.sz = s->s_iz; d.nt = s->nt;
        d.wav_off = wav_total;
        wav_total += s->nt + 1;
        d.wmap_off = wells;
        wells += P[b].nwells;
        d.seis_off = seis_total;
        seis_total += (long long)s->r_n * s->nt;
    }
    for (auto &d : desc) d.tshift = d.nt - ntmax;
    // per-shot well maps, wavelets and descriptors, concatenated
    std::vector<int> wcol((size_t)nb * ctx->ntx), wmap((size_t)wells * ctx->ldz);
    std::vector<float> wav(wav_total, 0.f);
    for (int b = 0; b < nb; b++) {
        std::copy(P[b].wcol.begin(), P[b].wcol.end(), wcol.begin() + (size_t)b * ctx->ntx);
        std::copy(P[b].wmap.begin(), P[b].wmap.end(), wmap.begin() + (size_t)desc[b].wmap_off * ctx->ldz);
        std::vector<float> r;
        CKR(host_copy(ctx, r, ricks[idx[b]], desc[b].nt));
        std::copy(r.begin(), r.end(), wav.begin() + desc[b].wav_off);
    }
    CKR(ensure(ctx, ctx->bat.wcol, sizeof(int) * wcol.size()));
    CKR(ensure(ctx, ctx->bat.wmap, sizeof(int) * std::max<size_t>(wmap.size(), 1)));
    CKR(ensure(ctx, ctx->bat.desc, sizeof(ShotDesc) * nb));
    CKR(ensure(ctx, ctx->bat.wav, sizeof(float) * wav.size()));
    CK(cudaMemcpyAsync(ctx->bat.wcol.p, wcol.data(), sizeof(int) * wcol.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->bat.wmap.p, wmap.data(), sizeof(int) * wmap.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->bat.desc.p, desc.data(), sizeof(ShotDesc) * nb, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->bat.wav.p, wav.data(), sizeof(float) * wav.size(), cudaMemcpyHostToDevice, ctx->stream));
    // receiver data: raw traces, then -int int dt dt (or a copy) into the injected traces,
    // which sit at the start of the buffer so the captured graphs see the same pointer
    CKR(ensure(ctx, ctx->bat.rdata, sizeof(float) * 2 * seis_total));
    float *rms = F(ctx->bat.rdata), *raw = rms + seis_total;
    for (int b = 0; b < nb; b++) {
        const swd_shot *s = &shots[idx[b]];
        const size_t n = (size_t)s->r_n * s->nt;
        CKR(to_dev(ctx, raw + desc[b].seis_off, data[idx[b]], sizeof(float) * n));
        if (flags & SWD_RTM_PREPROCESS) {
            k_preprocess<<<(s->r_n + 127) / 128, 128, 0, ctx->stream>>>(raw + desc[b].seis_off, rms + desc[b].seis_off,
                                                                        s->r_n, s->nt, ctx->grid.dt);
            ctx->launches++;
        } else {
            CK(cudaMemcpyAsync(rms + desc[b].seis_off, raw + desc[b].seis_off, sizeof(float) * n,
                               cudaMemcpyDeviceToDevice, ctx->stream));
        }
    }
    CK(cudaGetLastError());
    // zeroed state: source and receiver wavefields, dp/dt, FP64 images
    for (auto &w : ctx->bat.w)
        for (auto &b : w) CKR(ensure_bgrid(ctx, b, sizeof(float), nb));
    CKR(ensure_bgrid(ctx, ctx->bat.dpdt, sizeof(float), nb));
    CKR(ensure_bgrid(ctx, ctx->bat.I, sizeof(double), nb));
    CKR(ensure_bgrid(ctx, ctx->bat.S, sizeof(double), nb));
    if (ctx->image_blocks) {
        CKR(ensure_bgrid(ctx, ctx->bat.Ip, sizeof(float), nb));
        CKR(ensure_bgrid(ctx, ctx->bat.Sp, sizeof(float), nb));
    }
    // boundary strips: [shot][nt_max][slen] (+ scales [shot][nt_max][nscale] at 16 bits); the
    // per-shot stride uses the context's nt_max so every batch shares one captured graph
    const dim3 grid2 = grid_blocks(ctx);
    const dim3 grid(grid2.x, grid2.y, nb);
    const int slen = strip_len(ctx), nscale = grid2.x * grid2.y;
    const int ntcap = ctx->grid.nt_max;
    const size_t esz = ctx->strip_prec == SWD_STRIP_F32 ? 4 : 2;
    const size_t sbytes = ((size_t)ntcap * slen * esz + 255) / 256 * 256;
    CKR(ensure(ctx, ctx->bat.strips, sbytes * nb));
    if (ctx->strip_prec != SWD_STRIP_F32) CKR(ensure(ctx, ctx->bat.scale, sizeof(float) * (size_t)ntcap * nscale * nb));
    Batch bt;
    bt.desc = (const ShotDesc *)ctx->bat.desc.p;
    bt.bstride = (long long)batch_stride(ctx);
    bt.strip_bytes = (long long)sbytes;
    bt.scale_stride = (long long)ntcap * nscale;
    bt.nshots = nb;
    Strips st;
    st.buf = ctx->bat.strips.p;
    st.scale = ctx->strip_prec != SWD_STRIP_F32 ? F(ctx->bat.scale) : nullptr;
    st.slen = slen;
    st.prec = ctx->strip_prec;
    st.nscale = nscale;
    CKR(ensure(ctx, ctx->ctrl, 64));
    // forward: strips saved, nothing recorded
    FwdArgs a;
    memset(&a, 0, sizeof a);
    a.g = make_geo(ctx);
    a.c = make_cpml(ctx);
    a.vp = F(ctx->vp);
    a.rho = F(ctx->rho);
    a.m = make_mat(ctx);
    a.w[0] = a.w[1] = batch_wave(ctx, 0);
    a.itp = I32(ctx->ctrl);
    a.wav0 = a.wav1 = F(ctx->bat.wav);
    a.wells.wcol = I32(ctx->bat.wcol);
    a.wells.wmap = I32(ctx->bat.wmap);
    a.strips = st;
    a.s0_mod = 1;
    a.bt = bt;
    const int nf = probe_steps > 0 ? std::min(probe_steps, ntmax) : ntmax;
    {
        auto launch = [&](int k, cudaEvent_t *ev) {
            FwdArgs q = a;
            q.itoff = k;
            LC_DISPATCH(ctx->Lc, launch_fwd_batch, q, grid, ctx->stream, ev);
        };
        const int kid[2] = {0, 1};
        CKR(run_steps(ctx, ctx->gbf, &a, sizeof a, 0, +1, nf, 2, kid, launch));
    }
    // backward: reconstruction + receiver back-propagation + FP64 imaging, per-shot time index
    BwdArgs bb;
    memset(&bb, 0, sizeof bb);
    bb.g = a.g;
    bb.c = a.c;
    bb.vp = a.vp;
    bb.rho = a.rho;
    bb.m = a.m;
    bb.s = batch_wave(ctx, 0);
    bb.r = batch_wave(ctx, 1);
    bb.dpdt = F(ctx->bat.dpdt);
    bb.itp = I32(ctx->ctrl);
    bb.wavsub = F(ctx->bat.wav);
    bb.strips = st;
    bb.wells = a.wells;
    bb.rdata = rms;
    bb.I = D(ctx->bat.I);
    bb.S = D(ctx->bat.S);
    bb.Ip = ctx->image_blocks ? F(ctx->bat.Ip) : nullptr;
    bb.Sp = ctx->image_blocks ? F(ctx->bat.Sp) : nullptr;
    bb.bt = bt;
    const int nbk = probe_steps > 0 ? std::min(probe_steps, ntmax - 1) : ntmax - 1;
    {
        const int by_kind = ctx->bwd_by_kind;
        auto launch = [&](int k, cudaEvent_t *ev) {
            BwdArgs q = bb;
            q.itoff = -k;
            LC_DISPATCH(ctx->Lc, launch_bwd_batch, q, grid, ctx->stream, ev, by_kind);
        };
        const int kid[2] = {2, 3};
        std::vector<char> key((const char *)&bb, (const char *)&bb + sizeof bb);
        key.insert(key.end(), (const char *)&by_kind, (const char *)&by_kind + sizeof by_kind);
        CKR(run_steps(ctx, ctx->gbb, key.data(), key.size(), ntmax - 2, -1, nbk, 2, kid, launch));
    }
    if (probe_steps > 0) return SWD_OK;
    // per-shot normalisation, -vp^2 Laplacian and FP64 stack
    const size_t nimg = (size_t)ctx->nx * ctx->nz;
    if (!ctx->stack.p) {
        CKR(ensure(ctx, ctx->stack, sizeof(double) * nimg));
        CK(cudaMemsetAsync(ctx->stack.p, 0, sizeof(double) * nimg, ctx->stream));
    }
    CKR(ensure(ctx, ctx->bat.reduce, sizeof(unsigned long long) * nb));
    CK(cudaMemsetAsync(ctx->bat.reduce.p, 0, sizeof(unsigned long long) * nb, ctx->stream));
    const size_t gb = (size_t)ctx->ntx * ctx->ldz;
    for (int b = 0; b < nb; b++) {
        const double *I = D(ctx->bat.I) + (size_t)b * batch_stride(ctx);
        const double *S = D(ctx->bat.S) + (size_t)b * batch_stride(ctx);
        unsigned long long *mx = (unsigned long long *)ctx->bat.reduce.p + b;
        k_max_nonneg<<<592, 256, 0, ctx->stream>>>(S, gb, mx);
        k_rtm_post<<<dim3((ctx->nz + 31) / 32, (ctx->nx + 7) / 8), dim3(32, 8), 0, ctx->stream>>>(
            I, S, F(ctx->vp), mx, ctx->ntx, ctx->ntz, ctx->ldz, ctx->pmlc, ctx->grid.dx, ctx->grid.dz, nullptr, nullptr,
            nullptr, D(ctx->stack));
        ctx->launches += 2;
    }
    CK(cudaGetLastError());
    return SWD_OK;
}

// Batch size by measurement: for B in 1, 2, 4, 8 (up to the number of shots and half the
// free device memory), run a probe of 2 graph chunks forward and backward on the first B
// shots twice and keep the B with the least time per shot of the second run.
static int batch_autotune(swd_ctx *ctx, const swd_shot *shots, const float *const *ricks, const float *const *data,
                          const int *order, int nshots, unsigned flags, int *best)
{
    const int probe = 2 * GRAPH_K;
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    const size_t esz = ctx->strip_prec == SWD_STRIP_F32 ? 4 : 2;
    const size_t per_shot = batch_stride(ctx) * (14 * 4 + 4 + 16) + (size_t)ctx->grid.nt_max * strip_len(ctx) * esz;
    double best_t = 0.0;
    int choice = 1;
    cudaEvent_t e0 = ev_get(ctx), e1 = ev_get(ctx);
    int rc = SWD_OK;
    for (int B = 1; B <= 8 && B <= nshots && rc == SWD_OK; B *= 2) {
        if (B > 1 && (size_t)B * per_shot > free_b / 2) break;
        float ms = 0.f;
        for (int rep = 0; rep < 2 && rc == SWD_OK; rep++) {
            cudaEventRecord(e0, ctx->stream);
            rc = rtm_batch_run(ctx, shots, ricks, data, order, B, flags, probe);
            cudaEventRecord(e1, ctx->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
                rc = fail(ctx, SWD_ERR_CUDA, "batch autotune timing failed");
        }
        const double per = ms / (double)B;
        if (rc == SWD_OK && (B == 1 || per < best_t)) { best_t = per; choice = B; }
    }
    ctx->ev_pool.push_back(e0);
    ctx->ev_pool.push_back(e1);
    *best = choice;
    return rc;
}

extern "C" {

int swd_rtm_batch(swd_ctx *ctx, int nshots, const swd_shot *shots, const float *const *ricks, const float *const *data,
                  unsigned flags)
{
    CKR(check_ready(ctx));
    if (nshots < 0 || (nshots > 0 && (!shots || !ricks || !data))) return fail(ctx, SWD_ERR_ARG, "bad batch");
    if (flags & (SWD_RTM_ILLUM_RCV | SWD_RTM_NO_STACK))
        return fail(ctx, SWD_ERR_ARG, "swd_rtm_batch stacks every shot; ILLUM_RCV / NO_STACK apply to swd_rtm_shot");
    for (int i = 0; i < nshots; i++)
        if (!ricks[i] || !data[i]) return fail(ctx, SWD_ERR_ARG, "shot %d has no wavelet or data", i);
    {   // every shot checked before any device work: an argument error leaves the stack as it was
        ShotPlan P;
        for (int i = 0; i < nshots; i++) CKR(plan_shot_host(ctx, &shots[i], P));
    }
    if (nshots == 0) return SWD_OK;
    // longest records first, so each batch's records end close together
    std::vector<int> order(nshots);
    for (int i = 0; i < nshots; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return shots[a].nt > shots[b].nt; });
    int B = ctx->batch_opt;
    if (B <= 0) {
        if (ctx->batch_tuned <= 0) CKR(batch_autotune(ctx, shots, ricks, data, order.data(), nshots, flags, &ctx->batch_tuned));
        B = ctx->batch_tuned;
    }
    for (int g = 0; g < nshots; g += B)
        CKR(rtm_batch_run(ctx, shots, ricks, data, order.data() + g, std::min(B, nshots - g), flags, 0));
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
    return SWD_OK;
}

int swd_set_option(swd_ctx *ctx, int option, int value)
{
    if (!ctx) return SWD_ERR_ARG;
    switch (option) {
        case SWD_OPT_GRAPHS:
            if (value != 0 && value != 1) return fail(ctx, SWD_ERR_ARG, "SWD_OPT_GRAPHS takes 0 or 1");
            ctx->use_graphs = value;
            return SWD_OK;
        case SWD_OPT_BATCH:
            if (value < 0 || value > 64) return fail(ctx, SWD_ERR_ARG, "SWD_OPT_BATCH takes 0 (autotune) .. 64");
            ctx->batch_opt = value;
            return SWD_OK;
        case SWD_OPT_IMAGE_BLOCKS:
            if (value != 0 && value != 1) return fail(ctx, SWD_ERR_ARG, "SWD_OPT_IMAGE_BLOCKS takes 0 or 1");
            ctx->image_blocks = value;
            return SWD_OK;
        case SWD_OPT_BWD_BY_KIND:
            if (value != 0 && value != 1) return fail(ctx, SWD_ERR_ARG, "SWD_OPT_BWD_BY_KIND takes 0 or 1");
            ctx->bwd_by_kind = value;
            return SWD_OK;
        case SWD_OPT_TMA:
            if (value != 0 && value != 1) return fail(ctx, SWD_ERR_ARG, "SWD_OPT_TMA takes 0 or 1");
            ctx->use_tma = value;
            return SWD_OK;
        case SWD_OPT_PDL:
            if (value != 0 && value != 1) return fail(ctx, SWD_ERR_ARG, "SWD_OPT_PDL takes 0 or 1");
            ctx->use_pdl = value;
            return SWD_OK;
        case SWD_OPT_STAGED:
            if (value != 0 && value != 1) return fail(ctx, SWD_ERR_ARG, "SWD_OPT_STAGED takes 0 or 1");
            ctx->use_staged = value;
            return SWD_OK;
        case SWD_OPT_AUTOTUNE:
            if (value != 0 && value != 1) return fail(ctx, SWD_ERR_ARG, "SWD_OPT_AUTOTUNE takes 0 or 1");
            ctx->autotune = value;
            // forward: bit 1 TMA-staged velocity launch, bit 2 fully staged pressure launch,
            // bits 8 / 16 the pressure kernel bounded to 4 / 6 blocks per SM, bit 32 the velocity
            // kernel bounded to 6 (stencil order 4); backward: bit 1 TMA-staged velocity launch,
            // bit 4 the reference's pairing, bits 8 / 16 the pressure-and-imaging kernel bounded to
            // 4 / 6 blocks per SM, bit 32 the velocity kernel bounded to 6 (stencil order 4)
            if (ctx->Lc == 4) {
                tune_reset(ctx->tfwd, {0, 32, 1, 2, 3, 8, 16});
                tune_reset(ctx->tbwd, {0, 32, 1, 4, 8, 16});
            } else {
                tune_reset(ctx->tfwd, {0, 1, 2, 3});
                tune_reset(ctx->tbwd, {0, 1, 4});
            }
            return SWD_OK;
        case SWD_OPT_LEAN:
            if (value != 0 && value != 1) return fail(ctx, SWD_ERR_ARG, "SWD_OPT_LEAN takes 0 or 1");
            ctx->use_lean = value;
            return SWD_OK;
        default:
            return fail(ctx, SWD_ERR_ARG, "unknown option %d", option);
    }
}

int swd_get_option(swd_ctx *ctx, int option, int *value)
{
    if (!ctx || !value) return SWD_ERR_ARG;
    switch (option) {
        case SWD_OPT_GRAPHS: *value = ctx->use_graphs; return SWD_OK;
        case SWD_OPT_BATCH: *value = ctx->batch_opt; return SWD_OK;
        case SWD_OPT_BATCH_TUNED: *value = ctx->batch_tuned; return SWD_OK;
        case SWD_OPT_IMAGE_BLOCKS: *value = ctx->image_blocks; return SWD_OK;
        case SWD_OPT_BWD_BY_KIND: *value = ctx->bwd_by_kind; return SWD_OK;
        case SWD_OPT_TMA: *value = ctx->use_tma; return SWD_OK;
        case SWD_OPT_PDL: *value = ctx->use_pdl; return SWD_OK;
        case SWD_OPT_STAGED: *value = ctx->use_staged; return SWD_OK;
        case SWD_OPT_AUTOTUNE: *value = ctx->autotune; return SWD_OK;
        case SWD_OPT_LEAN: *value = ctx->use_lean; return SWD_OK;
        case SWD_OPT_TUNED_FWD: *value = ctx->autotune && ctx->tfwd.choice >= 0 ? ctx->tfwd.cand[ctx->tfwd.choice] : -1; return SWD_OK;
        case SWD_OPT_TUNED_BWD: *value = ctx->autotune && ctx->tbwd.choice >= 0 ? ctx->tbwd.cand[ctx->tbwd.choice] : -1; return SWD_OK;
        default: return fail(ctx, SWD_ERR_ARG, "unknown option %d", option);
    }
}

}  // extern "C"
