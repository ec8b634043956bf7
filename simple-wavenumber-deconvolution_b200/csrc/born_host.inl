// born_host.inl -- host side of Born modelling and its exact adjoint (part of swd.cu's
// translation unit: it uses the context, the chunked-graph runner and the forward pass).
//
// Background S0 (the p-update sum of the unperturbed field) feeds both directions: the Born
// pass computes it on the fly beside the scattered field; the adjoint pass needs it in
// reverse step order, from full storage (every == 0) or by recomputing each segment of
// `every` steps from a state checkpoint.  All time loops are chunked CUDA graphs; a
// segment's forward recompute and its adjoint steps are one graph replay each.

template <int LC>
static void launch_adj(const AdjArgs &a, dim3 grid, cudaStream_t s, cudaEvent_t *ev)
{
    if (ev) cudaEventRecordWithFlags(ev[0], s, cudaEventRecordExternal);
    k_adj_v<LC><<<grid, dim3(32, 8), 0, s>>>(a);
    if (ev) { cudaEventRecordWithFlags(ev[1], s, cudaEventRecordExternal); cudaEventRecordWithFlags(ev[2], s, cudaEventRecordExternal); }
    k_adj_p<LC><<<grid, dim3(32, 8), 0, s>>>(a);
    if (ev) cudaEventRecordWithFlags(ev[3], s, cudaEventRecordExternal);
}

static int ckpt_snapshots(const swd_ctx *c, int nt) { return c->ckpt_every > 0 ? (nt + c->ckpt_every - 1) / c->ckpt_every : 0; }

// checkpoint store layout: data [snap][7][ntx*ldz] then, for 16-bit, scales [snap][7][nblocks]
static size_t ckpt_layout(swd_ctx *c, int nt, void *base, Ckpt *ck)
{
    const dim3 grid = grid_blocks(c);
    const int nsnap = ckpt_snapshots(c, nt);
    const size_t fstride = (size_t)c->ntx * c->ldz;
    const size_t esz = c->ckpt_prec == SWD_STRIP_F32 ? 4 : 2;
    const size_t data = ((size_t)nsnap * 7 * fstride * esz + 255) / 256 * 256;
    const size_t nblocks = (size_t)grid.x * grid.y;
    const size_t scales = c->ckpt_prec == SWD_STRIP_F32 ? 0 : (size_t)nsnap * 7 * nblocks * sizeof(float);
    if (ck) {
        memset(ck, 0, sizeof *ck);
        ck->buf = base;
        ck->scale = scales ? (float *)((char *)base + data) : nullptr;
        ck->every = c->ckpt_every;
        ck->prec = c->ckpt_prec;   // SWD_STRIP_* values are the device codes
        ck->nblocks = (int)nblocks;
        ck->fstride = (long long)fstride;
    }
    return nsnap ? data + scales : 0;
}

// forward-step arguments of one background (+ optional scattered) field, no strips
static FwdArgs born_fwd_args(swd_ctx *ctx, const swd_shot *s, bool twin)
{
    FwdArgs a;
    memset(&a, 0, sizeof a);
    a.g = make_geo(ctx);
    a.c = make_cpml(ctx);
    a.vp = F(ctx->vp);
    a.rho = F(ctx->rho);
    a.m = make_mat(ctx);
    a.w[0] = make_wave(ctx, 0);
    a.w[1] = twin ? make_wave(ctx, 1) : make_wave(ctx, 0);
    a.sx = s->s_ix;
    a.sz = s->s_iz;
    a.nt = s->nt;
    a.wells.wcol = I32(ctx->wcol);
    a.wells.wmap = I32(ctx->wmap);
    a.itp = I32(ctx->ctrl);
    a.wav0 = F(ctx->wav);
    a.wav1 = F(ctx->wav) + s->nt;
    a.s0_stride = (long long)ctx->ntx * ctx->ldz;
    a.s0_mod = 1;
    return a;
}

// steps [t0, t0+n) of the background field alone, S0 into slot it % s0_mod
static int born_recompute(swd_ctx *ctx, const FwdArgs &base, int t0, int n, int klen)
{
    const dim3 grid = grid_blocks(ctx);
    auto launch = [&](int k, cudaEvent_t *ev) {
        FwdArgs b = base;
        b.itoff = k;
        if (ev) cudaEventRecordWithFlags(ev[0], ctx->stream, cudaEventRecordExternal);
        LC_DISPATCH(ctx->Lc, launch_fwd_v, b, 1, grid, ctx->stream);
        if (ev) { cudaEventRecordWithFlags(ev[1], ctx->stream, cudaEventRecordExternal); cudaEventRecordWithFlags(ev[2], ctx->stream, cudaEventRecordExternal); }
        LC_DISPATCH(ctx->Lc, launch_fwd_p, b, 1, grid, ctx->stream);
        if (ev) cudaEventRecordWithFlags(ev[3], ctx->stream, cudaEventRecordExternal);
    };
    const int kid[2] = {0, 1};
    FwdArgs key = base;
    key.itoff = 0;
    return run_steps(ctx, ctx->gseg, &key, sizeof key, t0, +1, n, 2, kid, launch, klen);
}

// adjoint steps t1-1 down to t1-n
static int born_adjoint_steps(swd_ctx *ctx, const AdjArgs &base, int t1, int n, int klen)
{
    const dim3 grid = grid_blocks(ctx);
    auto launch = [&](int k, cudaEvent_t *ev) {
        AdjArgs q = base;
        q.itoff = -k;
        LC_DISPATCH(ctx->Lc, launch_adj, q, grid, ctx->stream, ev);
    };
    const int kid[2] = {8, 9};
    AdjArgs key = base;
    key.itoff = 0;
    return run_steps(ctx, ctx->gadj, &key, sizeof key, t1 - 1, -1, n, 2, kid, launch, klen, 10);
}

static int zero_grid(swd_ctx *ctx, DevBuf &b, size_t elem)
{
    CKR(ensure_grid(ctx, b, elem));
    CK(cudaMemsetAsync(b.p, 0, b.n, ctx->stream));
    return SWD_OK;
}

extern "C" {

int swd_set_checkpointing(swd_ctx *ctx, int every, int prec)
{
    if (!ctx) return SWD_ERR_ARG;
    if (every < 0) return fail(ctx, SWD_ERR_ARG, "checkpoint interval %d < 0", every);
    if (prec < SWD_STRIP_F32 || prec > SWD_STRIP_I16) return fail(ctx, SWD_ERR_ARG, "unknown checkpoint precision %d", prec);
    ctx->ckpt_every = every;
    ctx->ckpt_prec = prec;
    return SWD_OK;
}

int swd_checkpoint_bytes(swd_ctx *ctx, int nt, size_t *bytes)
{
    if (!ctx || !bytes || nt < 1) return fail(ctx, SWD_ERR_ARG, "swd_checkpoint_bytes: bad arguments");
    *bytes = ckpt_layout(ctx, nt, nullptr, nullptr);
    return SWD_OK;
}

// a caller checkpoint buffer must be device memory of at least the layout's size
static int check_ckpt(swd_ctx *ctx, const swd_shot *shot, const void *ckpt, size_t bytes)
{
    if (!ckpt || ctx->ckpt_every == 0) return SWD_OK;
    if (!is_device_ptr_on(ckpt, ctx->dev)) return fail(ctx, SWD_ERR_ARG, "ckpt must be device memory of the context's GPU");
    if (!shot || shot->nt < 1) return fail(ctx, SWD_ERR_ARG, "shot is NULL or empty");
    const size_t need = ckpt_layout(ctx, shot->nt, nullptr, nullptr);
    if (bytes < need) return fail(ctx, SWD_ERR_ARG, "ckpt holds %zu bytes, %zu needed", bytes, need);
    return SWD_OK;
}

int swd_born(swd_ctx *ctx, const swd_shot *shot, const float *rick, const float *dkappa, float *dseis, void *ckpt,
             size_t ckpt_bytes)
{
    CKR(check_ready(ctx));
    if (!rick || !dkappa || !dseis) return fail(ctx, SWD_ERR_ARG, "rick, dkappa and dseis are required");
    CKR(check_ckpt(ctx, shot, ckpt, ckpt_bytes));
    ShotPlan P;
    CKR(plan_shot(ctx, shot, P));
    const int nt = shot->nt, r_n = shot->r_n;
    CKR(ensure_grid(ctx, ctx->dk, sizeof(float)));
    CKR(grid_to_dev(ctx, F(ctx->dk), dkappa));
    FwdJob J;
    J.shot = shot;
    CKR(host_copy(ctx, J.rick, rick, nt));
    J.twin = true;
    J.dkappa = F(ctx->dk);
    if (ckpt && ctx->ckpt_every > 0) ckpt_layout(ctx, nt, ckpt, &J.ck);
    CKR(ensure(ctx, ctx->seis, sizeof(float) * (size_t)r_n * nt));
    CK(cudaMemsetAsync(ctx->seis.p, 0, sizeof(float) * (size_t)r_n * nt, ctx->stream));
    J.seis_dev = F(ctx->seis);
    CKR(run_forward(ctx, J, P));
    CKR(copy_aliases(ctx, P, F(ctx->seis), nt));
    CKR(from_dev(ctx, dseis, ctx->seis.p, sizeof(float) * (size_t)r_n * nt));
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
    return SWD_OK;
}

int swd_born_adjoint(swd_ctx *ctx, const swd_shot *shot, const float *rick, const float *resid, double *grad,
                     const void *ckpt, size_t ckpt_bytes)
{
    CKR(check_ready(ctx));
    if (!rick || !resid || !grad) return fail(ctx, SWD_ERR_ARG, "rick, resid and grad are required");
    CKR(check_ckpt(ctx, shot, ckpt, ckpt_bytes));
    ShotPlan P;
    CKR(plan_shot(ctx, shot, P));
    const int nt = shot->nt, r_n = shot->r_n;
    const size_t ntr = (size_t)r_n * nt;
    const size_t fstride = (size_t)ctx->ntx * ctx->ldz;
    const int every = ctx->ckpt_every;
    ctx->kept.valid = false;   // wave[0] and wave[1] are reused below
    // adjoint source: residual traces, duplicates of a cell summed into the injected trace
    CKR(ensure(ctx, ctx->rbuf, sizeof(float) * ntr));
    CKR(to_dev(ctx, ctx->rbuf.p, resid, sizeof(float) * ntr));
    std::vector<int2> al;
    for (auto &a : P.alias)
        if (a.first != a.second) al.push_back(make_int2(a.first, a.second));
    if (!al.empty()) {
        CKR(ensure(ctx, ctx->alias, sizeof(int2) * al.size()));
        CK(cudaMemcpyAsync(ctx->alias.p, al.data(), sizeof(int2) * al.size(), cudaMemcpyHostToDevice, ctx->stream));
        k_sum_aliases<<<(nt + 255) / 256, 256, 0, ctx->stream>>>(F(ctx->rbuf), (const int2 *)ctx->alias.p, (int)al.size(), nt);
        ctx->launches++;
        CK(cudaGetLastError());
    }
    FwdJob J;
    J.shot = shot;
    CKR(host_copy(ctx, J.rick, rick, nt));
    CKR(ensure(ctx, ctx->ctrl, 64));
    // background: full S0 storage, or checkpoints (given, or taken by a pass here)
    Ckpt ck{};
    const int slots = every > 0 ? every : nt;
    CKR(ensure(ctx, ctx->s0, sizeof(float) * fstride * slots));
    if (every == 0) {
        J.s0 = F(ctx->s0);
        J.s0_mod = nt;
        CKR(run_forward(ctx, J, P));
    } else if (ckpt) {
        ckpt_layout(ctx, nt, (void *)ckpt, &ck);
        CKR(zero_wave(ctx, 0));   // allocated; every segment restores its state
        CKR(upload_wavelets(ctx, J, nt));
    } else {
        const size_t bytes = ckpt_layout(ctx, nt, nullptr, nullptr);
        CKR(ensure(ctx, ctx->ckpt, bytes));
        ckpt_layout(ctx, nt, ctx->ckpt.p, &ck);
        J.ck = ck;
        CKR(run_forward(ctx, J, P));
    }
    // adjoint state (wavefield 1), scratch and gradient start at zero
    CKR(zero_wave(ctx, 1));
    for (auto &b : ctx->adj) CKR(zero_grid(ctx, b, sizeof(float)));
    CKR(zero_grid(ctx, ctx->gk, sizeof(double)));
    AdjArgs b;
    memset(&b, 0, sizeof b);
    b.g = make_geo(ctx);
    b.c = make_cpml(ctx);
    b.vp = F(ctx->vp);
    b.rho = F(ctx->rho);
    b.ck = F(ctx->mat[2]);
    b.l = make_wave(ctx, 1);
    b.qx = F(ctx->adj[0]); b.qz = F(ctx->adj[1]); b.rx = F(ctx->adj[2]); b.rz = F(ctx->adj[3]);
    b.itp = I32(ctx->ctrl);
    b.nt = nt;
    b.wells.wcol = I32(ctx->wcol);
    b.wells.wmap = I32(ctx->wmap);
    b.resid = F(ctx->rbuf);
    b.s0 = F(ctx->s0);
    b.s0_stride = (long long)fstride;
    b.s0_mod = slots;
    b.grad = D(ctx->gk);
    if (every == 0) {
        CKR(born_adjoint_steps(ctx, b, nt, nt, GRAPH_K));
    } else {
        FwdArgs f = born_fwd_args(ctx, shot, false);
        f.s0_out = F(ctx->s0);
        f.s0_mod = every;
        const dim3 grid = grid_blocks(ctx);
        for (int c = ckpt_snapshots(ctx, nt) - 1; c >= 0; c--) {
            const int t0 = c * every, t1 = std::min(nt, t0 + every);
            k_ckpt_restore<<<grid, dim3(32, 8), 0, ctx->stream>>>(ck, make_wave(ctx, 0), c, ctx->ntx, ctx->ntz, ctx->ldz);
            ctx->launches++;
            CK(cudaGetLastError());
            CKR(born_recompute(ctx, f, t0, t1 - t0, every));
            CKR(born_adjoint_steps(ctx, b, t1, t1 - t0, every));
        }
    }
    CK(cudaGetLastError());
    CK(cudaMemcpy2DAsync(grad, ctx->ntz * sizeof(double), D(ctx->gk), ctx->ldz * sizeof(double), ctx->ntz * sizeof(double),
                         ctx->ntx, is_device_ptr(grad) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
    return SWD_OK;
}

}  // extern "C"
