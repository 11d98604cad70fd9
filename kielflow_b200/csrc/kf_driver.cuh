// kf_driver.cuh -- the reference's time loop around the step (kielflow.cpp:
// 172-182, 277-340): the density's log/linear transforms and the slice /
// backup output cadence, with the output fields formed on the device and
// copied to pinned host buffers on a side stream while later steps run.
//
// Included by kf_capi.cu after the forward driver (uses kf_ctx, the
// standalone transform passes, rk4_step and the step graph).

namespace {

struct OutState {
    double *O[5] = {};     // device, FP64: FUx, FUy, FUz, Fn (linear n), FPh
    double *H[2][5] = {};  // pinned host, double-buffered
    cudaStream_t st = nullptr;
    cudaEvent_t ready = nullptr, copied[2] = {};
};

void out_release(kf_ctx *c) {
    OutState *o = c->out;
    if (!o) return;
    for (auto &hb : o->H)
        for (double *h : hb)
            if (h) cudaFreeHost(h);
    if (o->ready) cudaEventDestroy(o->ready);
    for (auto e : o->copied)
        if (e) cudaEventDestroy(e);
    if (o->st) cudaStreamDestroy(o->st);
    delete o;  // device buffers are in c->allocs
    c->out = nullptr;
}

void out_init(kf_ctx *c) {
    if (c->out) return;
    c->out = new OutState;
    OutState &o = *c->out;
    const size_t bytes = 16 * (size_t)c->Nc;
    for (int q = 0; q < 5; ++q) o.O[q] = dalloc<double>(c, bytes);
    for (int b = 0; b < 2; ++b)
        for (int q = 0; q < 5; ++q) CK(cudaMallocHost(&o.H[b][q], bytes));
    CK(cudaStreamCreateWithFlags(&o.st, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&o.ready, cudaEventDisableTiming));
    for (auto &e : o.copied) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

// bulk-precision complex field -> FP64 device buffer (2 Nc doubles)
void to_f64(kf_ctx *c, double *dst, const void *src) {
    const long M = 2 * c->Nc;
    if (!c->fp32) {
        CK(cudaMemcpyAsync(dst, src, 8 * M, cudaMemcpyDeviceToDevice, c->st));
    } else {
        Launch L_(c, KC_MISC, 12. * M);
        k_to_f64<float><<<nblk(M, 256), 256, 0, c->st>>>(dst, (const float *)src, M);
    }
}

void explog(kf_ctx *c, void *x, int fn) {
    Launch L_(c, KC_MISC, 2. * c->es * c->N);
    if (c->fp32)
        k_explog<float><<<nblk(c->N, 256), 256, 0, c->st>>>((float *)x, fn, c->N);
    else
        k_explog<double><<<nblk(c->N, 256), 256, 0, c->st>>>((double *)x, fn, c->N);
}

// The fields save_slice / save_all receive (kielflow.cpp:290-324), on the
// device: the state's u' spectra, Fn = r2c(exp(c2r(s^))) and FPh = r2c(phi)
// (phi of the last stage solve, as the reference's Ph).  Work buffers CX[0],
// R[0] (and the standalone transforms' intermediates) are free between steps.
void out_fields(kf_ctx *c) {
    OutState &o = *c->out;
    for (int q = 0; q < 3; ++q) to_f64(c, o.O[q], c->Y[q]);
    CK(cudaMemcpyAsync(c->CX[0], c->Y[3], c->cs * c->Nc, cudaMemcpyDeviceToDevice, c->st));
    c->c2r_fn(c);
    explog(c, c->R[0], 0);
    c->r2c_fn(c);
    to_f64(c, o.O[3], c->CX[0]);
    if (c->fp32) {
        Launch L_(c, KC_MISC, 12. * c->N);
        k_from_f64<float><<<nblk(c->N, 256), 256, 0, c->st>>>((float *)c->R[0], c->phi, c->N);
    } else {
        CK(cudaMemcpyAsync(c->R[0], c->phi, 8 * c->N, cudaMemcpyDeviceToDevice, c->st));
    }
    c->r2c_fn(c);
    to_f64(c, o.O[4], c->CX[0]);
    CK(cudaGetLastError());
}

struct Pending {
    int step, kind, buf;
    double t;
};

void deliver(kf_ctx *c, const Pending &p, kf_output_fn fn, void *user) {
    OutState &o = *c->out;
    CK(cudaEventSynchronize(o.copied[p.buf]));
    if (!fn) return;
    kf_output out;
    out.step = p.step;
    out.t = p.t;
    out.kind = p.kind;
    out.FUx = o.H[p.buf][0];
    out.FUy = o.H[p.buf][1];
    out.FUz = o.H[p.buf][2];
    out.Fn = o.H[p.buf][3];
    out.FPh = o.H[p.buf][4];
    fn(&out, user);
}

void run_loop(kf_ctx *c, int iterations, double dt, double t0, int slice_every, int backup_every, kf_output_fn fn,
              void *user) {
    if (iterations < 0 || slice_every < 0 || backup_every < 0)
        throw KfError{KF_ERR_ARG, "kf_run: iterations, slice_every and backup_every must be >= 0"};
    out_init(c);
    OutState &o = *c->out;
    const bool g = graph_path(c);
    if (g) graph_begin(c, dt);
    std::vector<Pending> pend;
    int i_output = 0, i_backup = 0;  // counter.hpp: start at 0, output when they reach the limit
    double t_total = t0;
    int nout = 0;
    for (int step = 0; step < iterations; ++step) {
        if (g)
            graph_step(c);
        else
            rk4_step(c, dt, nullptr, nullptr, nullptr);
        int kind = 0;
        if (slice_every > 0 && i_output >= slice_every) {
            kind |= KF_OUT_SLICE;
            i_output = 0;
        }
        if (backup_every > 0 && i_backup >= backup_every) {
            kind |= KF_OUT_BACKUP;
            i_backup = 0;
        }
        if (kind) {
            const int b = nout % 2;
            if (pend.size() == 2) {  // host buffer b still holds output nout - 2
                deliver(c, pend.front(), fn, user);
                pend.erase(pend.begin());
            }
            // the device buffers hold output nout - 1 until its copy is done
            if (nout > 0) CK(cudaStreamWaitEvent(c->st, o.copied[(nout - 1) % 2], 0));
            out_fields(c);
            CK(cudaEventRecord(o.ready, c->st));
            CK(cudaStreamWaitEvent(o.st, o.ready, 0));
            for (int q = 0; q < 5; ++q)
                CK(cudaMemcpyAsync(o.H[b][q], o.O[q], 16 * c->Nc, cudaMemcpyDeviceToHost, o.st));
            CK(cudaEventRecord(o.copied[b], o.st));
            pend.push_back(Pending{step, kind, b, t_total});
            ++nout;
        }
        ++i_output;
        ++i_backup;
        t_total += dt;
    }
    for (const Pending &p : pend) deliver(c, p, fn, user);
    if (g)
        graph_end(c);
    else
        CK(cudaStreamSynchronize(c->st));
}

}  // namespace

extern "C" {

int kf_set_state_linear(kf_ctx *c, const double *ux, const double *uy, const double *uz, const double *n) {
    return guarded(c, [&] {
        if (!ux || !uy || !uz || !n) throw KfError{KF_ERR_ARG, "null state array"};
        const double *src[3] = {ux, uy, uz};
        for (int q = 0; q < 3; ++q) put_bulk(c, c->Y[q], src[q], 2 * c->Nc);
        put_bulk(c, c->CX[0], n, 2 * c->Nc);
        c->c2r_fn(c);
        explog(c, c->R[0], 1);
        c->r2c_fn(c);
        CK(cudaMemcpyAsync(c->Y[3], c->CX[0], c->cs * c->Nc, cudaMemcpyDeviceToDevice, c->st));
        copy_state(c, c->Ys, c->Y);
        c->nhist = 0;
        CK(cudaStreamSynchronize(c->st));
    });
}

int kf_get_output(kf_ctx *c, double *ux, double *uy, double *uz, double *n, double *phihat) {
    return guarded(c, [&] {
        out_init(c);
        out_fields(c);
        double *dst[5] = {ux, uy, uz, n, phihat};
        for (int q = 0; q < 5; ++q)
            if (dst[q]) CK(cudaMemcpyAsync(dst[q], c->out->O[q], 16 * c->Nc, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
    });
}

int kf_run(kf_ctx *c, int iterations, double dt, double t0, int slice_every, int backup_every, kf_output_fn fn,
           void *user) {
    return guarded(c, [&] { run_loop(c, iterations, dt, t0, slice_every, backup_every, fn, user); });
}

}  // extern "C"
