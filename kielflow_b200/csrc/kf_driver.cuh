// kf_driver.cuh -- the reference's time loop around the step (kielflow.cpp:
// 172-182, 277-340): the density's log/linear transforms and the slice /
// backup output cadence, with the output fields formed on the device and
// copied to pinned host buffers on a side stream while later steps run.
//
// Included by kf_capi.cu after the forward driver (uses kf_ctx, the
// standalone transform passes, rk4_step and the step graph).

#include <ctime>
#include <iomanip>
#include <sstream>

#include <unistd.h>

#include "kf_io.hpp"

std::string &kf_global_error();  // message of the last failure without a context (kf_capi.cu)

namespace {

struct OutState {
    double *O[5] = {};     // device, FP64: FUx, FUy, FUz, Fn (linear n), FPh
    double *H[2][5] = {};  // pinned host, double-buffered
    double *P[5] = {};     // device: real-space z = 0 planes (slice files)
    double *HP[2][5] = {}; // pinned host planes
    double *F[5] = {};     // device: real-space fields (backup files), on first use
    double *HF[5] = {};    // pinned host, on first use
    cudaStream_t st = nullptr;
    cudaEvent_t ready = nullptr, copied[2] = {};
};

void out_release(kf_ctx *c) {
    OutState *o = c->out;
    if (!o) return;
    for (auto &hb : o->H)
        for (double *h : hb)
            if (h) cudaFreeHost(h);
    for (auto &hb : o->HP)
        for (double *h : hb)
            if (h) cudaFreeHost(h);
    for (double *h : o->HF)
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
    const size_t pbytes = 8 * (size_t)c->n * c->n;
    for (int q = 0; q < 5; ++q) o.P[q] = dalloc<double>(c, pbytes);
    for (int b = 0; b < 2; ++b)
        for (int q = 0; q < 5; ++q) CK(cudaMallocHost(&o.HP[b][q], pbytes));
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

// z index of the slice plane: axis_CoEqSt::index_at(0.) = N*(0 - l0)/L
// (axis_EqSt.cpp:63-66), in the same double arithmetic
int slice_index(kf_ctx *c) {
    const double L = c->cfg.L, l0 = -0.5 * L;
    return (int)(c->n * (0. - l0) / L);
}

// real-space file fields of the current state into o.P (planes) or o.F (grid)
void real_fields(kf_ctx *c, bool plane) {
    OutState &o = *c->out;
    if (!plane && !o.F[0])
        for (int q = 0; q < 5; ++q) o.F[q] = dalloc<double>(c, 8 * (size_t)c->N);
    double *const *d = plane ? o.P : o.F;
    c->inv_state_fn(c);  // R[20..23] = c2r of the state
    const long M = plane ? (long)c->n * c->n : c->N;
    const int k0 = plane ? slice_index(c) : -1;
    Launch L_(c, KC_MISC, (4. * c->es + 8. + 40.) * M);
    if (c->fp32)
        k_out_real<float><<<nblk(M, 256), 256, 0, c->st>>>((const float *)c->R[20], (const float *)c->R[21],
                                                          (const float *)c->R[22], (const float *)c->R[23], c->phi,
                                                          d[0], d[1], d[2], d[3], d[4], c->n, k0, M);
    else
        k_out_real<double><<<nblk(M, 256), 256, 0, c->st>>>((const double *)c->R[20], (const double *)c->R[21],
                                                           (const double *)c->R[22], (const double *)c->R[23],
                                                           c->phi, d[0], d[1], d[2], d[3], d[4], c->n, k0, M);
    CK(cudaGetLastError());
}

std::string self_path() {
    char buf[4096];
    const ssize_t k = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
    return k > 0 ? std::string(buf, (size_t)k) : std::string();
}

// IO.cpp save_all / save_slice: the file's datasets in the reference's order
void write_file(kf_ctx *c, const std::string &path, double t, bool plane, double *const *f) {
    const kf_config &cf = c->cfg;
    kfio::File F;
    F.str("version", "kielflow_b200");
    F.i64("date", (int64_t)std::time(nullptr));
    F.str("path", self_path());
    for (const char *ax : {"x", "y", "z"}) {
        const std::string a(ax);
        F.i32("domain/type_" + a, c->stretched ? 3 : 1);  // axis_CoSiSt : axis_CoEqSt
        F.f64("domain/m_" + a, cf.stretch_m);
        F.f64("domain/l0_" + a, -0.5 * cf.L);
        F.i32("domain/N_" + a, c->n);
        F.f64("domain/L_" + a, cf.L);
    }
    F.f64("time", t);
    F.f64("parameters/mach number M", cf.M);
    F.f64("parameters/damping ratio tau", cf.tau);
    F.f64("parameters/temperature ratio theta", cf.theta);
    F.f64("parameters/velocity diffusion mu", cf.diff_D);
    F.f64("parameters/magnetization beta", 0.);
    const uint64_t n = (uint64_t)c->n;
    const char *names[5] = {"Ux", "Uy", "Uz", "ni", "Ph"};
    for (int q = 0; q < 5; ++q) {
        if (plane)
            F.array(std::string("data/") + names[q], {n, n}, f[q]);
        else
            F.array(std::string("data/") + names[q], {n, n, n}, f[q]);
    }
    std::string err;
    if (!F.write(path, err)) throw KfError{KF_ERR_ARG, err};
}

std::string slice_name(const std::string &dir, int step) {  // IO.cpp:1325 with I4()
    std::ostringstream s;
    s << dir << "/slice_" << std::setw(4) << std::setfill('0') << step << ".kfh";
    return s.str();
}

std::string backup_name(const std::string &dir, int step) {  // kielflow.cpp:319-320
    std::ostringstream s;
    s << dir << "/backup_at_" << step << ".kfh";
    return s.str();
}

struct Pending {
    int step, kind, buf;
    double t;
};

void deliver(kf_ctx *c, const Pending &p, kf_output_fn fn, void *user, const char *dir) {
    OutState &o = *c->out;
    CK(cudaEventSynchronize(o.copied[p.buf]));
    if (dir) {
        if (p.kind & KF_OUT_SLICE) write_file(c, slice_name(dir, p.step), p.t, true, o.HP[p.buf]);
        if (p.kind & KF_OUT_BACKUP) write_file(c, backup_name(dir, p.step), p.t, false, o.HF);
    }
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

void run_loop(kf_ctx *c, int iterations, double dt, double t0, int slice_every, int backup_every, const char *dir,
              kf_output_fn fn, void *user) {
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
            if (pend.size() == 2 || (dir && (kind & KF_OUT_BACKUP))) {
                // host buffer b still holds output nout - 2; the grid-sized
                // backup buffers are single: deliver what is pending first
                while (pend.size() > (dir && (kind & KF_OUT_BACKUP) ? 0u : 1u)) {
                    deliver(c, pend.front(), fn, user, dir);
                    pend.erase(pend.begin());
                }
            }
            // the device buffers hold output nout - 1 until its copy is done
            if (nout > 0) CK(cudaStreamWaitEvent(c->st, o.copied[(nout - 1) % 2], 0));
            out_fields(c);
            if (dir && (kind & KF_OUT_SLICE)) real_fields(c, true);
            if (dir && (kind & KF_OUT_BACKUP)) {
                real_fields(c, false);
                if (!o.HF[0])
                    for (int q = 0; q < 5; ++q) CK(cudaMallocHost(&o.HF[q], 8 * (size_t)c->N));
            }
            CK(cudaEventRecord(o.ready, c->st));
            CK(cudaStreamWaitEvent(o.st, o.ready, 0));
            for (int q = 0; q < 5; ++q)
                CK(cudaMemcpyAsync(o.H[b][q], o.O[q], 16 * c->Nc, cudaMemcpyDeviceToHost, o.st));
            if (dir && (kind & KF_OUT_SLICE))
                for (int q = 0; q < 5; ++q)
                    CK(cudaMemcpyAsync(o.HP[b][q], o.P[q], 8 * (size_t)c->n * c->n, cudaMemcpyDeviceToHost, o.st));
            if (dir && (kind & KF_OUT_BACKUP))
                for (int q = 0; q < 5; ++q)
                    CK(cudaMemcpyAsync(o.HF[q], o.F[q], 8 * (size_t)c->N, cudaMemcpyDeviceToHost, o.st));
            CK(cudaEventRecord(o.copied[b], o.st));
            pend.push_back(Pending{step, kind, b, t_total});
            ++nout;
        }
        ++i_output;
        ++i_backup;
        t_total += dt;
    }
    for (const Pending &p : pend) deliver(c, p, fn, user, dir);
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

int kf_run(kf_ctx *c, int iterations, double dt, double t0, int slice_every, int backup_every, const char *out_dir,
           kf_output_fn fn, void *user) {
    return guarded(c, [&] { run_loop(c, iterations, dt, t0, slice_every, backup_every, out_dir, fn, user); });
}

// frontend.cpp:255-330 (create_input_from_MGsolver and what follows) on the
// context's grid: phi from 0 with rho = n_background + n_d (the reference:
// n_background = 0), n = exp(-theta phi), both filtered by exp(-2000 k~^15)
// in k-space, u' = 0; the state takes s^ = r2c(log n) as kielflow.cpp:172-182
// does on loading the file.
int kf_frontend_state(kf_ctx *c, double n_background) {
    return guarded(c, [&] {
        const long N = c->N, Nc = c->Nc;
        CK(cudaMemsetAsync(c->phi, 0, 8 * N, c->st));
        {
            Launch L_(c, KC_MISC, 16. * N);
            k_add_const<<<nblk(N, 256), 256, 0, c->st>>>(c->rho, c->nd, n_background, N);
        }
        if (poisson(c)) throw KfError{KF_ERR_NOT_CONVERGED, "frontend Poisson solve did not reach its tolerance"};
        auto filter = [&]() {  // CX[0] *= PF
            Launch L_(c, KC_MISC, (2. * c->cs + c->es) * Nc);
            if (c->fp32)
                k_filter<float><<<nblk(Nc, 256), 256, 0, c->st>>>((float2 *)c->CX[0], (const float *)c->PF, Nc);
            else
                k_filter<double><<<nblk(Nc, 256), 256, 0, c->st>>>((double2 *)c->CX[0], (const double *)c->PF, Nc);
        };
        {
            Launch L_(c, KC_MISC, (8. + c->es) * N);
            if (c->fp32)
                k_boltzmann<float><<<nblk(N, 256), 256, 0, c->st>>>((float *)c->R[0], c->phi, c->cfg.theta, N);
            else
                k_boltzmann<double><<<nblk(N, 256), 256, 0, c->st>>>((double *)c->R[0], c->phi, c->cfg.theta, N);
        }
        c->r2c_fn(c);
        filter();
        c->c2r_fn(c);
        explog(c, c->R[0], 1);
        c->r2c_fn(c);
        CK(cudaMemcpyAsync(c->Y[3], c->CX[0], c->cs * Nc, cudaMemcpyDeviceToDevice, c->st));
        if (c->fp32) {
            Launch L_(c, KC_MISC, 12. * N);
            k_from_f64<float><<<nblk(N, 256), 256, 0, c->st>>>((float *)c->R[0], c->phi, N);
        } else {
            CK(cudaMemcpyAsync(c->R[0], c->phi, 8 * N, cudaMemcpyDeviceToDevice, c->st));
        }
        c->r2c_fn(c);
        filter();
        c->c2r_fn(c);
        if (c->fp32) {
            Launch L_(c, KC_MISC, 12. * N);
            k_to_f64<float><<<nblk(N, 256), 256, 0, c->st>>>(c->phi, (const float *)c->R[0], N);
        } else {
            CK(cudaMemcpyAsync(c->phi, c->R[0], 8 * N, cudaMemcpyDeviceToDevice, c->st));
        }
        for (int q = 0; q < 3; ++q) CK(cudaMemsetAsync(c->Y[q], 0, c->cs * Nc, c->st));
        copy_state(c, c->Ys, c->Y);
        c->nhist = 0;
        CK(cudaStreamSynchronize(c->st));
        CK(cudaGetLastError());
    });
}

int kf_save(kf_ctx *c, const char *path, int kind, double t) {
    return guarded(c, [&] {
        if (!path || (kind != KF_FILE_SLICE && kind != KF_FILE_BACKUP)) throw KfError{KF_ERR_ARG, "kf_save: path, kind"};
        out_init(c);
        OutState &o = *c->out;
        const bool plane = kind == KF_FILE_SLICE;
        real_fields(c, plane);
        const size_t cnt = plane ? (size_t)c->n * c->n : (size_t)c->N;
        std::vector<std::vector<double>> h(5, std::vector<double>(cnt));
        double *f[5];
        for (int q = 0; q < 5; ++q) {
            CK(cudaMemcpyAsync(h[q].data(), plane ? o.P[q] : o.F[q], 8 * cnt, cudaMemcpyDeviceToHost, c->st));
            f[q] = h[q].data();
        }
        CK(cudaStreamSynchronize(c->st));
        write_file(c, path, t, plane, f);
    });
}

int kf_file_info_read(const char *path, kf_file_info *info) {
    if (!path || !info) {
        kf_global_error() = "kf_file_info_read: null argument";
        return KF_ERR_ARG;
    }
    kfio::File F;
    std::string err;
    if (!F.read(path, err)) {
        kf_global_error() = err;
        return KF_ERR_ARG;
    }
    int32_t n = 0;
    kf_file_info r{};
    bool ok = F.get_i32("domain/N_x", n) && F.get_f64("domain/L_x", r.L) && F.get_f64("domain/l0_x", r.l0) &&
              F.get_f64("time", r.time) && F.get_f64("parameters/mach number M", r.M) &&
              F.get_f64("parameters/damping ratio tau", r.tau) &&
              F.get_f64("parameters/temperature ratio theta", r.theta) &&
              F.get_f64("parameters/velocity diffusion mu", r.mu) &&
              F.get_f64("parameters/magnetization beta", r.beta);
    const kfio::Entry *ux = F.find("data/Ux");
    if (!ok || !ux) {
        kf_global_error() = std::string(path) + ": missing domain, parameters, time or data";
        return KF_ERR_ARG;
    }
    r.n = n;
    r.kind = ux->dims.size() == 2 ? KF_FILE_SLICE : KF_FILE_BACKUP;
    int32_t type = 1;
    r.m = 0.;
    F.get_i32("domain/type_x", type);
    r.type = type;
    F.get_f64("domain/m_x", r.m);
    *info = r;
    return KF_OK;
}

int kf_load(kf_ctx *c, const char *path, double *t_out) {
    return guarded(c, [&] {
        if (!path) throw KfError{KF_ERR_ARG, "kf_load: null path"};
        kfio::File F;
        std::string err;
        if (!F.read(path, err)) throw KfError{KF_ERR_ARG, err};
        for (const char *ax : {"x", "y", "z"}) {
            int32_t n = 0, type = 1;
            double L = 0., m = 0.;
            F.get_i32(std::string("domain/type_") + ax, type);
            F.get_f64(std::string("domain/m_") + ax, m);
            if (!F.get_i32(std::string("domain/N_") + ax, n) || !F.get_f64(std::string("domain/L_") + ax, L) ||
                n != c->n || std::fabs(L - c->cfg.L) > 1e-12 * c->cfg.L || type != (c->stretched ? 3 : 1) ||
                std::fabs(m - c->cfg.stretch_m) > 1e-12 * c->cfg.L)
                throw KfError{KF_ERR_ARG, std::string(path) + ": grid differs from the context's"};
        }
        const char *names[5] = {"Ux", "Uy", "Uz", "ni", "Ph"};
        const kfio::Entry *e[5];
        for (int q = 0; q < 5; ++q) {
            e[q] = F.find(std::string("data/") + names[q]);
            if (!e[q] || e[q]->type != kfio::F64 || e[q]->count() != (size_t)c->N)
                throw KfError{KF_ERR_ARG, std::string(path) + ": data/" + names[q] + " is not a full real field"};
        }
        double t = 0.;
        if (!F.get_f64("time", t)) throw KfError{KF_ERR_ARG, std::string(path) + ": no time"};
        // u'_c = r2c(U_c); s = r2c(log n); phi = Ph
        for (int q = 0; q < 4; ++q) {
            put_bulk(c, c->R[0], (const double *)e[q]->data.data(), c->N);
            if (q == 3) explog(c, c->R[0], 1);
            c->r2c_fn(c);
            CK(cudaMemcpyAsync(c->Y[q], c->CX[0], c->cs * c->Nc, cudaMemcpyDeviceToDevice, c->st));
            CK(cudaStreamSynchronize(c->st));  // the host source of put_bulk is reused
        }
        CK(cudaMemcpyAsync(c->phi, e[4]->data.data(), 8 * c->N, cudaMemcpyHostToDevice, c->st));
        copy_state(c, c->Ys, c->Y);
        c->nhist = 0;
        CK(cudaStreamSynchronize(c->st));
        if (t_out) *t_out = t;
    });
}

}  // extern "C"
