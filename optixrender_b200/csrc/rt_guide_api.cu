// rt_guide_api.cu - C ABI of the path-guiding network (rt_guide_* in
// rt_capi.h): parameters, forward, gradients and Adam steps on host buffers.
// The renderer drives the same kernels on device buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "rt_guide_host.h"
#include "rt_internal.h"

using namespace rti;

namespace rtgh {

void level_resolutions(int n_max, int* res) {
    const double lo = std::min(16.0, double(n_max));
    const double b = std::exp((std::log(double(n_max)) - std::log(lo)) / double(rtg::kLevels - 1));
    for (int l = 0; l < rtg::kLevels; l++) res[l] = int(std::floor(lo * std::pow(b, double(l)) + 1e-6));
}

}  // namespace rtgh

struct rt_guide {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    rt_guide_options opt{};
    DevBuf table, table16, mlp, mlp16, gtable, gmlp, mt, vt, mm, vm, loss;
    DevBuf frags;  // training fragments of up to kFragTiles tiles, allocated at the first training pass
    int step = 0;
    int res[rtg::kLevels];
    int64_t used_entries[rtg::kLevels] = {};  // per level: entries any resolution so far has addressed
};

// Level resolutions for n_max, and the entries each level addresses: a dense
// level (res + 1)^3 of them, a hashed one the whole table.  The Adam update
// covers the largest count seen, so entries that once had a gradient keep
// their moments decaying after a resolution change.
static void set_resolutions(rt_guide* g, int n_max) {
    rtgh::level_resolutions(n_max, g->res);
    for (int l = 0; l < rtg::kLevels; l++) {
        const int64_t r1 = int64_t(g->res[l]) + 1;
        const int64_t n = r1 * r1 * r1 <= int64_t(rtg::kT) ? r1 * r1 * r1 : int64_t(rtg::kT);
        g->used_entries[l] = std::max(g->used_entries[l], n);
    }
}

namespace {

#define GD_CUDA(call, what)                                  \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(e_, what);   \
    } while (0)

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
float uniform(uint64_t& s) { return float(splitmix(s) >> 40) * (1.0f / 16777216.0f); }

// Training passes run in chunks of up to 2^18 samples (16,384 tiles, 235 MB
// of fragments).
constexpr int kFragTiles = 1 << 14;

rt_status ensure_frags(rt_guide* g) {
    if (g->frags.ptr) return RT_OK;
    GD_CUDA(g->frags.alloc(size_t(kFragTiles) * rtgh::frag_bytes_per_tile()), "allocate training fragments");
    return RT_OK;
}

rtg::NetView view(const rt_guide* g) {
    rtg::NetView v;
    v.table = g->table16.as<__half2>();
    v.mlp = g->mlp16.as<__half>();
    v.lo = make_float3(0.f, 0.f, 0.f);
    v.inv_ext = make_float3(1.f, 1.f, 1.f);
    for (int l = 0; l < rtg::kLevels; l++) v.res[l] = g->res[l];
    v.kappa_hi = g->opt.max_log_kappa;
    return v;
}

rt_status refresh_half(rt_guide* g) {
    rtgh::launch_to_half(g->table.as<float>(), g->table16.as<__half>(), rtg::kTableParams, g->stream);
    rtgh::launch_to_half(g->mlp.as<float>(), g->mlp16.as<__half>(), rtg::kMlpParams, g->stream);
    GD_CUDA(cudaGetLastError(), "guide: fp16 copy");
    return RT_OK;
}

rt_status upload(rt_guide* g, DevBuf& b, const float* src, int64_t n, const char* what) {
    GD_CUDA(b.alloc(size_t(n) * 4), what);
    GD_CUDA(cudaMemcpyAsync(b.ptr, src, size_t(n) * 4, cudaMemcpyHostToDevice, g->stream), what);
    return RT_OK;
}

}  // namespace

namespace rti {

// Shared by the renderer: creates the network on the current device.
rt_status guide_create(const rt_guide_options* o, rt_guide** out) {
    rt_guide* g = new (std::nothrow) rt_guide();
    if (!g) return fail(RT_ERR_OUT_OF_MEMORY, "rt_guide_create: out of host memory");
    rt_guide_options_default(&g->opt);
    if (o) g->opt = *o;
    cudaError_t e = cudaGetDevice(&g->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, g->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete g;
        return cuda_fail(e, "rt_guide_create");
    }
    if (g->opt.max_resolution < 2 || g->opt.max_resolution > (1 << 20) || !(g->opt.max_log_kappa > rtg::kKappaLo)) {
        rt_guide_destroy(g);
        return fail(RT_ERR_INVALID_ARG, "rt_guide_create: max_resolution in [2, 2^20], max_log_kappa > -2");
    }
    set_resolutions(g, g->opt.max_resolution);
    rt_status st = RT_OK;
    auto check = [&](cudaError_t ce, const char* what) {
        if (st == RT_OK && ce != cudaSuccess) st = cuda_fail(ce, what);
    };
    check(rtgh::prepare_kernels(), "rt_guide_create: kernel attributes");
    const size_t tb = size_t(rtg::kTableParams) * 4, mb = size_t(rtg::kMlpParams) * 4;
    check(g->table.alloc(tb), "rt_guide_create: allocate");
    check(g->table16.alloc(tb / 2), "rt_guide_create: allocate");
    check(g->gtable.alloc(tb), "rt_guide_create: allocate");
    check(g->mt.alloc(tb), "rt_guide_create: allocate");
    check(g->vt.alloc(tb), "rt_guide_create: allocate");
    check(g->mlp.alloc(mb), "rt_guide_create: allocate");
    check(g->mlp16.alloc(mb / 2), "rt_guide_create: allocate");
    check(g->gmlp.alloc(mb), "rt_guide_create: allocate");
    check(g->mm.alloc(mb), "rt_guide_create: allocate");
    check(g->vm.alloc(mb), "rt_guide_create: allocate");
    check(g->loss.alloc(4), "rt_guide_create: allocate");
    if (st == RT_OK) {
        // table U(-1e-4, 1e-4); weights U(+-sqrt(6 / (fan_in + fan_out)))
        uint64_t s = g->opt.seed * 0x2545F4914F6CDD1Dull + 1;
        std::vector<float> t(size_t(rtg::kTableParams)), w(size_t(rtg::kMlpParams));
        for (auto& x : t) x = (2.0f * uniform(s) - 1.0f) * 1e-4f;
        const int shape[4][2] = {{rtg::kHid, rtg::kIn}, {rtg::kHid, rtg::kHid}, {rtg::kHid, rtg::kHid}, {rtg::kOut, rtg::kHid}};
        size_t off = 0;
        for (auto& sh : shape) {
            const float a = std::sqrt(6.0f / float(sh[0] + sh[1]));
            for (int i = 0; i < sh[0] * sh[1]; i++) w[off++] = (2.0f * uniform(s) - 1.0f) * a;
        }
        check(cudaMemcpyAsync(g->table.ptr, t.data(), tb, cudaMemcpyHostToDevice, g->stream), "rt_guide_create");
        check(cudaMemcpyAsync(g->mlp.ptr, w.data(), mb, cudaMemcpyHostToDevice, g->stream), "rt_guide_create");
        DevBuf* zero[] = {&g->gtable, &g->mt, &g->vt, &g->gmlp, &g->mm, &g->vm};
        for (DevBuf* b : zero) check(cudaMemsetAsync(b->ptr, 0, b->bytes, g->stream), "rt_guide_create");
        if (st == RT_OK) st = refresh_half(g);
        check(cudaStreamSynchronize(g->stream), "rt_guide_create");
    }
    if (st != RT_OK) {
        rt_guide_destroy(g);
        return st;
    }
    *out = g;
    return RT_OK;
}

rtg::NetView guide_view(const rt_guide* g, float3 lo, float3 inv_ext) {
    rtg::NetView v = view(g);
    v.lo = lo;
    v.inv_ext = inv_ext;
    return v;
}

// Gradient of `n` device samples (scale multiplies every weight) followed by
// one Adam step, all on `st`.
rt_status guide_train_device(rt_guide* g, const float* pos, const float* dir, const float* weight, int n, float scale,
                             const float* weight_sum, cudaStream_t st) {
    rt_status fs = ensure_frags(g);
    if (fs) return fs;
    GD_CUDA(cudaMemsetAsync(g->loss.ptr, 0, 4, st), "guide training step");
    rtgh::launch_backward(view(g), pos, dir, weight, n, scale, weight_sum, g->gtable.as<float>(), g->gmlp.as<float>(),
                          g->loss.as<float>(), g->frags.as<uint32_t>(), kFragTiles, g->sms, st);
    g->step++;
    rtgh::launch_adam_table(g->table.as<float>(), g->table16.as<__half>(), g->gtable.as<float>(), g->mt.as<float>(),
                            g->vt.as<float>(), g->used_entries, g->opt.learning_rate, g->step, st);
    rtgh::launch_adam(g->mlp.as<float>(), g->mlp16.as<__half>(), g->gmlp.as<float>(), g->mm.as<float>(),
                      g->vm.as<float>(), rtg::kMlpParams, g->opt.learning_rate, g->step, st);
    GD_CUDA(cudaGetLastError(), "guide training step");
    return RT_OK;
}

int guide_sms(const rt_guide* g) { return g->sms; }

int64_t guide_device_bytes(const rt_guide* g) {
    const DevBuf* bufs[] = {&g->table, &g->table16, &g->mlp, &g->mlp16, &g->gtable, &g->gmlp,
                            &g->mt, &g->vt, &g->mm, &g->vm, &g->loss, &g->frags};
    int64_t b = 0;
    for (const DevBuf* d : bufs) b += int64_t(d->bytes);
    if (!g->frags.ptr) b += int64_t(kFragTiles) * int64_t(rtgh::frag_bytes_per_tile());  // allocated at the first training pass
    return b;
}

}  // namespace rti

extern "C" {

void rt_guide_options_default(rt_guide_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->learning_rate = 1e-2f;
    o->max_resolution = 64;
    o->seed = 1;
    o->max_log_kappa = 4.0f;
}

rt_status rt_guide_create(const rt_guide_options* o, rt_guide** out) {
    if (!out) return fail(RT_ERR_INVALID_ARG, "rt_guide_create: out is NULL");
    return guide_create(o, out);
}

rt_status rt_guide_destroy(rt_guide* g) {
    if (!g) return RT_OK;
    if (g->stream) {
        cudaStreamSynchronize(g->stream);
        cudaStreamDestroy(g->stream);
    }
    delete g;
    return RT_OK;
}

void rt_guide_sizes(int64_t* table_params, int64_t* mlp_params) {
    if (table_params) *table_params = rtg::kTableParams;
    if (mlp_params) *mlp_params = rtg::kMlpParams;
}

rt_status rt_guide_get_params(const rt_guide* g, float* table, float* mlp) {
    if (!g) return fail(RT_ERR_INVALID_ARG, "rt_guide_get_params: NULL guide");
    if (table)
        GD_CUDA(cudaMemcpyAsync(table, g->table.ptr, g->table.bytes, cudaMemcpyDeviceToHost, g->stream), "get params");
    if (mlp) GD_CUDA(cudaMemcpyAsync(mlp, g->mlp.ptr, g->mlp.bytes, cudaMemcpyDeviceToHost, g->stream), "get params");
    GD_CUDA(cudaStreamSynchronize(g->stream), "get params");
    return RT_OK;
}

rt_status rt_guide_set_params(rt_guide* g, const float* table, const float* mlp) {
    if (!g) return fail(RT_ERR_INVALID_ARG, "rt_guide_set_params: NULL guide");
    if (table)
        GD_CUDA(cudaMemcpyAsync(g->table.ptr, table, g->table.bytes, cudaMemcpyHostToDevice, g->stream), "set params");
    if (mlp) GD_CUDA(cudaMemcpyAsync(g->mlp.ptr, mlp, g->mlp.bytes, cudaMemcpyHostToDevice, g->stream), "set params");
    rt_status st = refresh_half(g);
    if (st) return st;
    GD_CUDA(cudaStreamSynchronize(g->stream), "set params");
    return RT_OK;
}

// The inference kernels' bounded waits on the tensor cores, after a synchronize.
static rt_status tc_status(const char* what) {
    const int n = rtgh::take_tc_timeouts();
    if (n == 0) return RT_OK;
    return fail(RT_ERR_DEVICE_WATCHDOG, std::string(what) + ": " + std::to_string(n) +
                                            " inference blocks gave up waiting for their tensor-core work");
}

rt_status rt_guide_forward(rt_guide* g, const float* pos, int64_t n, float* raw) {
    if (!g || n < 0 || (n > 0 && (!pos || !raw)) || n > (int64_t(1) << 28))
        return fail(RT_ERR_INVALID_ARG, "rt_guide_forward: bad argument");
    if (n == 0) return RT_OK;
    DevBuf dp, dr;
    rt_status st = upload(g, dp, pos, n * 3, "rt_guide_forward");
    if (st) return st;
    GD_CUDA(dr.alloc(size_t(n) * rtg::kOut * 4), "rt_guide_forward");
    rtgh::launch_forward(view(g), dp.as<float>(), int(n), 0, dr.as<float>(), nullptr, g->sms, g->stream);
    GD_CUDA(cudaGetLastError(), "rt_guide_forward");
    GD_CUDA(cudaMemcpyAsync(raw, dr.ptr, dr.bytes, cudaMemcpyDeviceToHost, g->stream), "rt_guide_forward");
    GD_CUDA(cudaStreamSynchronize(g->stream), "rt_guide_forward");
    return tc_status("rt_guide_forward");
}

rt_status rt_guide_gradients(rt_guide* g, const float* pos, const float* dir, const float* weight, int64_t n,
                             float* loss, float* grad_table, float* grad_mlp) {
    if (!g || n <= 0 || !pos || !dir || !weight || n > (int64_t(1) << 28))
        return fail(RT_ERR_INVALID_ARG, "rt_guide_gradients: bad argument");
    DevBuf dp, dd, dw;
    rt_status st = upload(g, dp, pos, n * 3, "rt_guide_gradients");
    if (!st) st = upload(g, dd, dir, n * 3, "rt_guide_gradients");
    if (!st) st = upload(g, dw, weight, n, "rt_guide_gradients");
    if (st) return st;
    GD_CUDA(cudaMemsetAsync(g->gtable.ptr, 0, g->gtable.bytes, g->stream), "rt_guide_gradients");
    GD_CUDA(cudaMemsetAsync(g->gmlp.ptr, 0, g->gmlp.bytes, g->stream), "rt_guide_gradients");
    GD_CUDA(cudaMemsetAsync(g->loss.ptr, 0, 4, g->stream), "rt_guide_gradients");
    st = ensure_frags(g);
    if (st) return st;
    rtgh::launch_backward(view(g), dp.as<float>(), dd.as<float>(), dw.as<float>(), int(n), 1.0f / float(n), nullptr,
                          g->gtable.as<float>(), g->gmlp.as<float>(), g->loss.as<float>(), g->frags.as<uint32_t>(),
                          kFragTiles, g->sms, g->stream);
    GD_CUDA(cudaGetLastError(), "rt_guide_gradients");
    if (loss) GD_CUDA(cudaMemcpyAsync(loss, g->loss.ptr, 4, cudaMemcpyDeviceToHost, g->stream), "rt_guide_gradients");
    if (grad_table)
        GD_CUDA(cudaMemcpyAsync(grad_table, g->gtable.ptr, g->gtable.bytes, cudaMemcpyDeviceToHost, g->stream),
                "rt_guide_gradients");
    if (grad_mlp)
        GD_CUDA(cudaMemcpyAsync(grad_mlp, g->gmlp.ptr, g->gmlp.bytes, cudaMemcpyDeviceToHost, g->stream),
                "rt_guide_gradients");
    GD_CUDA(cudaMemsetAsync(g->gtable.ptr, 0, g->gtable.bytes, g->stream), "rt_guide_gradients");
    GD_CUDA(cudaMemsetAsync(g->gmlp.ptr, 0, g->gmlp.bytes, g->stream), "rt_guide_gradients");
    GD_CUDA(cudaStreamSynchronize(g->stream), "rt_guide_gradients");
    return RT_OK;
}

rt_status rt_guide_train_step(rt_guide* g, const float* pos, const float* dir, const float* weight, int64_t n,
                              float* loss) {
    if (!g || n <= 0 || !pos || !dir || !weight || n > (int64_t(1) << 28))
        return fail(RT_ERR_INVALID_ARG, "rt_guide_train_step: bad argument");
    double sum = 0.0;
    for (int64_t i = 0; i < n; i++) sum += double(weight[i]);
    if (!(sum > 0.0)) return fail(RT_ERR_INVALID_ARG, "rt_guide_train_step: weights sum to zero");
    DevBuf dp, dd, dw;
    rt_status st = upload(g, dp, pos, n * 3, "rt_guide_train_step");
    if (!st) st = upload(g, dd, dir, n * 3, "rt_guide_train_step");
    if (!st) st = upload(g, dw, weight, n, "rt_guide_train_step");
    if (st) return st;
    GD_CUDA(cudaMemsetAsync(g->loss.ptr, 0, 4, g->stream), "rt_guide_train_step");
    st = guide_train_device(g, dp.as<float>(), dd.as<float>(), dw.as<float>(), int(n), float(1.0 / sum), nullptr,
                            g->stream);
    if (st) return st;
    if (loss) GD_CUDA(cudaMemcpyAsync(loss, g->loss.ptr, 4, cudaMemcpyDeviceToHost, g->stream), "rt_guide_train_step");
    GD_CUDA(cudaStreamSynchronize(g->stream), "rt_guide_train_step");
    return RT_OK;
}

rt_status rt_guide_set_hyperparameters(rt_guide* g, float lr, int32_t max_resolution, float max_log_kappa) {
    if (!g) return fail(RT_ERR_INVALID_ARG, "rt_guide_set_hyperparameters: NULL guide");
    if (max_resolution > (1 << 20) || (max_resolution > 0 && max_resolution < 2) ||
        (max_log_kappa != 0.0f && !(max_log_kappa > rtg::kKappaLo)))
        return fail(RT_ERR_INVALID_ARG, "rt_guide_set_hyperparameters: max_resolution in [2, 2^20], max_log_kappa > -2");
    if (lr > 0.0f) g->opt.learning_rate = lr;
    if (max_resolution > 0) {
        g->opt.max_resolution = max_resolution;
        set_resolutions(g, max_resolution);
    }
    if (max_log_kappa != 0.0f) g->opt.max_log_kappa = max_log_kappa;
    return RT_OK;
}

rt_status rt_guide_last_loss(rt_guide* g, float* loss, int64_t* steps) {
    if (!g || !loss) return fail(RT_ERR_INVALID_ARG, "rt_guide_last_loss: NULL argument");
    GD_CUDA(cudaDeviceSynchronize(), "rt_guide_last_loss");
    GD_CUDA(cudaMemcpy(loss, g->loss.ptr, 4, cudaMemcpyDeviceToHost), "rt_guide_last_loss");
    if (steps) *steps = g->step;
    return RT_OK;
}

rt_status rt_guide_pdf(rt_guide* g, const float* pos, const float* dir, const float* u, int64_t n, float* out_dir,
                       float* pdf) {
    if (!g || n < 0 || (n > 0 && (!pos || !pdf || (!dir && !u) || (u && !out_dir))) || n > (int64_t(1) << 26))
        return fail(RT_ERR_INVALID_ARG, "rt_guide_pdf: bad argument");
    if (n == 0) return RT_OK;
    DevBuf dp, dd, du, dmix, dout, dpdf;
    rt_status st = upload(g, dp, pos, n * 3, "rt_guide_pdf");
    if (!st && dir && !u) st = upload(g, dd, dir, n * 3, "rt_guide_pdf");
    if (!st && u) st = upload(g, du, u, n * 3, "rt_guide_pdf");
    if (st) return st;
    GD_CUDA(dmix.alloc(size_t(n) * sizeof(rtg::Mixture)), "rt_guide_pdf");
    GD_CUDA(dpdf.alloc(size_t(n) * 4), "rt_guide_pdf");
    if (u) GD_CUDA(dout.alloc(size_t(n) * 12), "rt_guide_pdf");
    rtgh::launch_forward(view(g), dp.as<float>(), int(n), 1, nullptr, dmix.as<rtg::Mixture>(), g->sms, g->stream);
    rtgh::launch_pdf_sample(dmix.as<rtg::Mixture>(), dd.as<float>(), du.as<float>(), int(n), dout.as<float>(),
                            dpdf.as<float>(), g->stream);
    GD_CUDA(cudaGetLastError(), "rt_guide_pdf");
    GD_CUDA(cudaMemcpyAsync(pdf, dpdf.ptr, dpdf.bytes, cudaMemcpyDeviceToHost, g->stream), "rt_guide_pdf");
    if (u) GD_CUDA(cudaMemcpyAsync(out_dir, dout.ptr, dout.bytes, cudaMemcpyDeviceToHost, g->stream), "rt_guide_pdf");
    GD_CUDA(cudaStreamSynchronize(g->stream), "rt_guide_pdf");
    return tc_status("rt_guide_pdf");
}

}  // extern "C"
