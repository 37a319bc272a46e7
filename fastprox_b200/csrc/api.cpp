// The extern "C" boundary of libfastprox_b200: argument checks in the order
// of the reference's prox_impl (src/api/api.cpp:413-559), the device
// workspace (all device memory allocated at creation), the host loop that
// drives the per-iteration launches, and per-image results. No exception
// crosses the boundary (guard), as in the reference (src/api/api.cpp:28-38).
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <new>
#include <vector>

#include "../../include/fastprox_b200.h"
#include "engine.h"
#include "launch.h"
#include "pool.h"
#include "workspace.h"

using namespace fpb;

namespace {

constexpr double kMaxScaledStep = 0x1p960;  // the reference's step range (core/op.hpp:48)

template <class F>
fp_status guard(F &&f) noexcept {
    try {
        return f();
    } catch (const std::bad_alloc &) {
        return FP_ENOMEM;
    } catch (...) {
        return FP_EINTERNAL;
    }
}

bool finite_nonneg(double v) { return std::isfinite(v) && v >= 0.0; }

// A validated array descriptor (scalars become shape [1]).
struct Arr {
    char *data = nullptr;
    int dtype = 0;
    int ndim = 0;
    int device = 0;
    int64_t shape[FP_MAX_NDIM] = {};
    int64_t strides[FP_MAX_NDIM] = {};
    int64_t numel() const {
        int64_t n = 1;
        for (int d = 0; d < ndim; ++d) n *= shape[d];
        return n;
    }
    size_t itemsize() const { return dtype == FP_F32 || dtype == FP_I32 ? 4 : (dtype == FP_I8 ? 1 : 8); }
    bool contiguous() const {
        int64_t s = 1;
        for (int d = ndim - 1; d >= 0; --d) {
            if (shape[d] != 1 && strides[d] != s) return false;
            s *= shape[d];
        }
        return true;
    }
};

int enum_bits_dtype(const fp_array *a) {
    int v;
    std::memcpy(&v, &a->dtype, sizeof v);
    return v;
}
int enum_bits_device(const fp_array *a) {
    int v;
    std::memcpy(&v, &a->device, sizeof v);
    return v;
}

constexpr int64_t kMaxElems = (int64_t(1) << 60) - 1;

// The dtypes an array may have (src/api/api.cpp:54-56): float32 and float64
// (data), int8 (masks, states, signs, sides), int32 and int64 (labels).
enum class Dt { Float, Int8, Label };

// src/api/api.cpp:57-110: the dtype of its class, 0 <= ndim <= 32, extents
// >= 0, the entry count and offset span below 2^60.
fp_status to_arr(const fp_array *a, Arr &out, Dt kind = Dt::Float) {
    if (!a) return FP_EINVAL;
    const int dev = enum_bits_device(a);
    if (dev != FP_DEVICE_CPU && dev != FP_DEVICE_CUDA) return FP_EINVAL;
    const int dt = enum_bits_dtype(a);
    if (kind == Dt::Float && dt != FP_F32 && dt != FP_F64) return FP_EDTYPE;
    if (kind == Dt::Int8 && dt != FP_I8) return FP_EDTYPE;
    if (kind == Dt::Label && dt != FP_I32 && dt != FP_I64) return FP_EDTYPE;
    if (a->ndim < 0 || a->ndim > FP_MAX_NDIM) return FP_ESHAPE;
    out.data = static_cast<char *>(a->data);
    out.dtype = dt;
    out.device = dev;
    if (a->ndim == 0) {
        out.ndim = 1;
        out.shape[0] = 1;
        out.strides[0] = 1;
    } else {
        if (!a->shape) return FP_EINVAL;
        out.ndim = a->ndim;
        double count = 1.0;
        for (int d = 0; d < a->ndim; ++d) {
            if (a->shape[d] < 0) return FP_ESHAPE;
            out.shape[d] = a->shape[d];
            out.strides[d] = a->strides ? a->strides[d] : 0;
            if (a->shape[d] > 1) count *= (double)a->shape[d];
        }
        if (count > (double)kMaxElems) return FP_ESHAPE;
        if (!a->strides) {
            int64_t s = 1;
            for (int d = a->ndim - 1; d >= 0; --d) {
                out.strides[d] = s;
                s *= out.shape[d];
            }
        }
        double span = 0.0;
        for (int d = 0; d < a->ndim; ++d)
            if (out.shape[d] > 1) span += (double)(out.shape[d] - 1) * (double)std::llabs(out.strides[d]);
        if (span > (double)kMaxElems) return FP_ESHAPE;
    }
    if (!out.data && out.numel() > 0) return FP_EINVAL;
    return FP_OK;
}

// The lowest and highest byte an array touches.
void byte_range(const Arr &a, intptr_t &lo, intptr_t &hi) {
    intptr_t l = 0, h = 0;
    for (int d = 0; d < a.ndim; ++d) {
        if (a.shape[d] < 2) continue;
        const intptr_t e = (intptr_t)(a.shape[d] - 1) * (intptr_t)a.strides[d] * (intptr_t)a.itemsize();
        if (e < 0) l += e;
        else h += e;
    }
    lo = (intptr_t)a.data + l;
    hi = (intptr_t)a.data + h + (intptr_t)a.itemsize() - 1;
}

// src/api/api.cpp check_output: out may be x itself; any other overlap, or a
// stride 0 on an extent > 1 in out, is FP_EINVAL.
fp_status check_output(const Arr *x, const Arr &out) {
    if (out.numel() == 0) return FP_OK;
    for (int d = 0; d < out.ndim; ++d)
        if (out.shape[d] > 1 && out.strides[d] == 0) return FP_EINVAL;
    if (!x || out.numel() == 0 || x->numel() == 0) return FP_OK;
    bool same = x->data == out.data && x->ndim == out.ndim && x->dtype == out.dtype;
    for (int d = 0; same && d < x->ndim; ++d)
        same = x->shape[d] == out.shape[d] && (x->shape[d] < 2 || x->strides[d] == out.strides[d]);
    if (same) return FP_OK;
    intptr_t xl, xh, ol, oh;
    byte_range(*x, xl, xh);
    byte_range(out, ol, oh);
    return (oh < xl || ol > xh) ? FP_OK : FP_EINVAL;
}

bool same_shape(const Arr &a, const Arr &b) {
    if (a.ndim != b.ndim) return false;
    for (int d = 0; d < a.ndim; ++d)
        if (a.shape[d] != b.shape[d]) return false;
    return true;
}

// A one-dimensional host parameter array of any float dtype and stride.
fp_status read_vec(const fp_array *a, std::vector<double> &v) {
    v.clear();
    if (!a) return FP_OK;
    Arr x;
    if (fp_status s = to_arr(a, x)) return s;
    if (x.device != FP_DEVICE_CPU) return FP_EINVAL;
    if (a->ndim > 1) return FP_ESHAPE;
    const int64_t m = x.shape[0];
    if (m == 0) return FP_ESHAPE;
    v.resize((size_t)m);
    for (int64_t i = 0; i < m; ++i) {
        const char *p = x.data + i * x.strides[0] * (int64_t)x.itemsize();
        v[(size_t)i] = x.dtype == FP_F32 ? (double)*reinterpret_cast<const float *>(p) : *reinterpret_cast<const double *>(p);
    }
    return FP_OK;
}

// An n-d host parameter array of exactly nd axes, copied in C order.
fp_status read_nd(const fp_array *a, int nd, std::vector<double> &v, int64_t *shape) {
    Arr x;
    if (fp_status s = to_arr(a, x)) return s;
    if (x.device != FP_DEVICE_CPU) return FP_EINVAL;
    if (a->ndim != nd) return FP_ESHAPE;
    const int64_t n = x.numel();
    if (n == 0) return FP_ESHAPE;
    for (int d = 0; d < nd; ++d) shape[d] = x.shape[d];
    v.resize((size_t)n);
    std::vector<int64_t> idx((size_t)nd, 0);
    for (int64_t i = 0; i < n; ++i) {
        int64_t off = 0;
        for (int d = 0; d < nd; ++d) off += idx[(size_t)d] * x.strides[d];
        const char *p = x.data + off * (int64_t)x.itemsize();
        v[(size_t)i] = x.dtype == FP_F32 ? (double)*reinterpret_cast<const float *>(p) : *reinterpret_cast<const double *>(p);
        for (int d = nd - 1; d >= 0; --d) {
            if (++idx[(size_t)d] < x.shape[d]) break;
            idx[(size_t)d] = 0;
        }
    }
    return FP_OK;
}

fp_options defaults() {
    fp_options o;
    o.axis = -1;
    o.threads = 0;
    o.tol = 1e-6;
    o.max_iter = 1000;
    o.tie = 0;
    o.keep_structure = 0;
    return o;
}

// Restores the caller's current device on scope exit.
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceScope() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// The device an array lives on (-1: host or unknown).
int pointer_device(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) return at.device;
    return -1;
}

bool host_pinned(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

}  // namespace

// ---------------------------------------------------------------------------
// Operators
// ---------------------------------------------------------------------------

extern "C" {

FP_API void fp_options_init(fp_options *opt) {
    if (opt) *opt = defaults();
}

}  // extern "C"

namespace {

// tv_iso.cpp:1072-1095 and tv_aniso.cpp make_tv_aniso: the parameter rules.
fp_status make_tv(int kind, int ndim, const std::vector<double> &w, std::vector<double> spatial,
                  const int64_t *sshape, fp_op **out) {
    if (ndim != 2 && ndim != 3) return FP_EPARAM;
    double ww[3] = {1.0, 1.0, 1.0};
    if (w.size() == 1) {
        for (int a = 0; a < ndim; ++a) ww[a] = w[0];
    } else if (!w.empty()) {
        if ((int)w.size() != ndim) return FP_ESHAPE;
        for (int a = 0; a < ndim; ++a) ww[a] = w[(size_t)a];
    }
    for (int a = 0; a < ndim; ++a)
        if (!finite_nonneg(ww[a])) return FP_EPARAM;
    if (!spatial.empty()) {
        double n = 1.0;
        for (int a = 0; a < ndim; ++a) n *= (double)sshape[a];
        if (!(n < 2147483647.0)) return FP_ESHAPE;
        for (double v : spatial)
            if (!finite_nonneg(v)) return FP_EPARAM;
    }
    auto op = std::make_unique<fp_op>();
    op->kind = kind;
    op->k = ndim;
    for (int a = 0; a < 3; ++a) op->w[a] = a < ndim ? ww[a] : 0.0;
    op->spatial = std::move(spatial);
    for (int a = 0; a < 3; ++a) op->sshape[a] = (sshape && a < ndim) ? sshape[a] : 1;
    op->smax = 0.0;
    for (double v : op->spatial) op->smax = std::max(op->smax, v);
    *out = op.release();
    return FP_OK;
}

}  // namespace

extern "C" {

FP_API fp_status fp_op_tv_iso(int ndim, const fp_array *axis_weights, fp_op **out) {
    return guard([&] {
        if (!out) return FP_EINVAL;
        *out = nullptr;
        std::vector<double> w;
        if (fp_status s = read_vec(axis_weights, w)) return s;
        return make_tv(kIso, ndim, w, {}, nullptr, out);
    });
}

FP_API fp_status fp_op_tv_aniso(int ndim, const fp_array *axis_weights, fp_op **out) {
    return guard([&] {
        if (!out) return FP_EINVAL;
        *out = nullptr;
        std::vector<double> w;
        if (fp_status s = read_vec(axis_weights, w)) return s;
        return make_tv(kAniso, ndim, w, {}, nullptr, out);
    });
}

FP_API fp_status fp_op_tv_iso_weighted(int ndim, const fp_array *axis_weights, const fp_array *pixel_weights,
                                       fp_op **out) {
    return guard([&] {
        if (!out) return FP_EINVAL;
        *out = nullptr;
        if (!pixel_weights) return FP_EINVAL;
        if (ndim != 2 && ndim != 3) return FP_EPARAM;
        std::vector<double> w, al;
        int64_t shape[3] = {1, 1, 1};
        if (fp_status s = read_vec(axis_weights, w)) return s;
        if (fp_status s = read_nd(pixel_weights, ndim, al, shape)) return s;
        return make_tv(kIso, ndim, w, std::move(al), shape, out);
    });
}

FP_API fp_status fp_op_tv_aniso_weighted(int ndim, const fp_array *axis_weights, const fp_array *edge_weights,
                                         fp_op **out) {
    return guard([&] {
        if (!out) return FP_EINVAL;
        *out = nullptr;
        if (!edge_weights) return FP_EINVAL;
        if (ndim != 2 && ndim != 3) return FP_EPARAM;
        std::vector<double> w, b;
        int64_t shape[4] = {1, 1, 1, 1};
        if (fp_status s = read_vec(axis_weights, w)) return s;
        if (fp_status s = read_nd(edge_weights, ndim + 1, b, shape)) return s;
        if (shape[0] != ndim) return FP_ESHAPE;
        return make_tv(kAniso, ndim, w, std::move(b), shape + 1, out);
    });
}

FP_API void fp_op_free(fp_op *op) { delete op; }

FP_API int64_t fp_op_nparams(const fp_op *op) {
    if (!op) return 0;
    return op->k + (int64_t)op->spatial.size() + (op->huber ? 1 : 0);
}

FP_API const char *fp_op_name(const fp_op *op) {
    if (!op) return "";
    if (op->huber) return op->kind == kIso ? "tv_iso_huber" : "tv_aniso_huber";
    return op->kind == kIso ? "tv_iso" : "tv_aniso";
}

// Huber-smoothed TV: the TV operators' parameter rules and a smoothing delta,
// finite and > 0 (the Huber function's, fp_op_huber).
FP_API fp_status fp_b200_op_tv_iso_huber(int ndim, const fp_array *axis_weights, const fp_array *pixel_weights,
                                         double delta, fp_op **out) {
    return guard([&] {
        if (!out) return FP_EINVAL;
        *out = nullptr;
        if (!std::isfinite(delta) || !(delta > 0.0)) return FP_EPARAM;
        fp_status s = pixel_weights ? fp_op_tv_iso_weighted(ndim, axis_weights, pixel_weights, out)
                                    : fp_op_tv_iso(ndim, axis_weights, out);
        if (s == FP_OK) {
            (*out)->huber = true;
            (*out)->delta = delta;
        }
        return s;
    });
}

FP_API fp_status fp_b200_op_tv_aniso_huber(int ndim, const fp_array *axis_weights, const fp_array *edge_weights,
                                           double delta, fp_op **out) {
    return guard([&] {
        if (!out) return FP_EINVAL;
        *out = nullptr;
        if (!std::isfinite(delta) || !(delta > 0.0)) return FP_EPARAM;
        fp_status s = edge_weights ? fp_op_tv_aniso_weighted(ndim, axis_weights, edge_weights, out)
                                   : fp_op_tv_aniso(ndim, axis_weights, out);
        if (s == FP_OK) {
            (*out)->huber = true;
            (*out)->delta = delta;
        }
        return s;
    });
}

FP_API int fp_device_available(fp_device dev) {
    int n = 0;
    const int d = (int)dev;
    if (d != FP_DEVICE_CPU && d != FP_DEVICE_CUDA) return 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n > 0 ? 1 : 0;
}

FP_API fp_status fp_op_device_check(const fp_op *op, fp_device dev, int *row_parallel_only) {
    if (!op) return FP_EINVAL;
    if (row_parallel_only) *row_parallel_only = 0;
    return fp_device_available(dev) ? FP_OK : FP_EINVAL;
}

FP_API const char *fp_strerror(fp_status s) {
    switch ((int)s) {
    case FP_OK: return "success";
    case FP_EINVAL: return "invalid argument";
    case FP_EDTYPE: return "unsupported or mismatched dtype";
    case FP_ESHAPE: return "mismatched shapes or parameter lengths";
    case FP_ENOMEM: return "out of memory";
    case FP_ENOTCONV: return "iterative operator did not converge";
    case FP_EPARAM: return "invalid operator parameter or step";
    case FP_EINTERNAL: return "internal error";
    case FP_EDEVICE: return "device error";
    default: return "unknown status";
    }
}

FP_API int fp_abi_version(void) { return FP_ABI_VERSION; }
FP_API const char *fp_version_string(void) { return "1.0.6+b200"; }
FP_API int fp_default_threads(void) { return 1; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Workspaces
// ---------------------------------------------------------------------------

namespace {

void free_ws_memory(fp_workspace *ws) {
    DeviceScope ds(ws->device);
    pool_free(ws->device, ws->dev_block);
    ws->dev_block = nullptr;
    pinned_give(ws->host_block, ws->host_bytes);
    ws->host_block = nullptr;
    for (int i = 0; i < 2; ++i)
        if (ws->ev[i]) cudaEventDestroy(ws->ev[i]);
    ws->ev[0] = ws->ev[1] = nullptr;
    for (cudaEvent_t e : ws->tev) cudaEventDestroy(e);
    ws->tev.clear();
    if (ws->an_graph) cudaGraphExecDestroy(ws->an_graph);
    ws->an_graph = nullptr;
}

// The buffers of a workspace, laid out in one block (256-byte aligned
// pieces) before the block exists; place() points them into it.
struct Layout {
    std::vector<std::pair<void **, size_t>> parts;
    size_t total = 0;
    void add(void **p, size_t bytes) {
        *p = nullptr;
        parts.emplace_back(p, total);
        total += (std::max<size_t>(bytes, 16) + 255) / 256 * 256;
    }
    void place(void *base) const {
        for (const auto &pr : parts) *pr.first = static_cast<char *>(base) + pr.second;
    }
};

// The image plan of x: leading axes are the batch, the last k the image.
fp_status image_geometry(const fp_op &op, const Arr &x, Geometry &g) {
    const int k = op.k;
    if (x.ndim < k) return FP_ESHAPE;
    g.k = k;
    g.N = 1;
    for (int a = 0; a < 3; ++a) g.L[a] = 1;
    for (int a = 0; a < k; ++a) {
        g.L[a] = x.shape[x.ndim - k + a];
        g.N *= g.L[a];
    }
    g.B = 1;
    for (int d = 0; d < x.ndim - k; ++d) g.B *= x.shape[d];
    return FP_OK;
}

// tv_iso.cpp:170-177: 32-bit region labels, and the shape of spatial weights.
fp_status check_image(const fp_op &op, const Arr &x) {
    const int k = op.k;
    double n = 1.0;
    for (int a = 0; a < k; ++a) n *= (double)x.shape[x.ndim - k + a];
    if (!op.spatial.empty())
        for (int a = 0; a < k; ++a)
            if (x.shape[x.ndim - k + a] != op.sshape[a]) return FP_ESHAPE;
    return n < 2147483647.0 ? FP_OK : FP_ESHAPE;
}

fp_status cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return FP_OK;
    if (e == cudaErrorMemoryAllocation) return FP_ENOMEM;
    return FP_EDEVICE;
}

}  // namespace

fp_status fpb_workspace_build(const fp_op *op, const Arr &x, const fp_options &o, int device, fp_workspace **out) {
    Geometry g;
    if (fp_status s = image_geometry(*op, x, g)) return s;
    auto ws = std::make_unique<fp_workspace>();
    ws->op = op;
    ws->device = device;
    ws->dtype = x.dtype;
    ws->ndim = x.ndim;
    for (int d = 0; d < x.ndim; ++d) ws->shape[d] = x.shape[d];
    ws->g = g;
    ws->host_mode = x.device == FP_DEVICE_CPU;
    ws->keep = o.keep_structure != 0;
    DeviceScope dsc(device);
    const size_t T = x.dtype == FP_F32 ? 4 : 8;
    const int64_t B = std::max<int64_t>(g.B, 1), N = std::max<int64_t>(g.N, 1);
    const size_t img = (size_t)B * (size_t)N * T;
    const size_t dualb = img * (size_t)g.k;
    fp_status s = FP_OK;
    Layout dev, host;
    auto A = [&](void **p, size_t bytes) { dev.add(p, bytes); };
    A(&ws->d, img);
    A(&ws->stage, img);  // strided or conjugate inputs, strided outputs
    for (int i = 0; i < 2; ++i) {
        A(&ws->U[i], dualb);
        A(&ws->V[i], dualb);
    }
    A(&ws->dual, dualb);
    std::vector<char> spatial_h;
    if (!op->spatial.empty()) {
        A(&ws->spatial, op->spatial.size() * T);
        spatial_h.resize(op->spatial.size() * T);
        for (size_t i = 0; i < op->spatial.size(); ++i) {
            if (T == 4) reinterpret_cast<float *>(spatial_h.data())[i] = (float)op->spatial[i];
            else reinterpret_cast<double *>(spatial_h.data())[i] = op->spatial[i];
        }
    }
    // per-image state, partials and tickets; launch shape (tuning hints from
    // the environment: FASTPROX_B200_ROWS, FASTPROX_B200_BX, FASTPROX_B200_KIND=1 for the generic step)
    auto env_int = [](const char *n) {
        const char *v = std::getenv(n);
        return v ? std::atoi(v) : 0;
    };
    ws->shape_ = iso_pick_shape(x.dtype, g, env_int("FASTPROX_B200_ROWS"), env_int("FASTPROX_B200_BX"),
                                op->huber ? 1 : env_int("FASTPROX_B200_KIND"));
    if (const int ch = env_int("FASTPROX_B200_CHUNK")) ws->chunk = ch;
    ws->max_part = std::max(iso_setup_blocks(g), ws->shape_.gx * ws->shape_.gy);
    ws->max_part = std::max(ws->max_part, 4096);
    if (ws->shape_.kind == 4)  // per-row partial sums of the lean 2D step
        ws->max_part = (int)std::max<int64_t>(ws->max_part, (int64_t)ws->shape_.gx * g.L[0]);
    if (x.dtype == FP_F32 && g.k == 2 && !op->huber)  // per-row, per-strip partial sums of the quad launch
        ws->max_part = (int)std::max<int64_t>(ws->max_part, iso_quad_parts(g));
    if (op->kind == kAniso && !op->huber) {
        // the untiled fibre passes: a block of 128 fibres per partial, three
        // axes in one launch for FDPG-3
        int64_t nfmax = 0;
        for (int a = 0; a < g.k; ++a) nfmax = std::max<int64_t>(nfmax, g.N / std::max<int64_t>(g.L[a], 1));
        ws->max_part = (int)std::max<int64_t>(ws->max_part, 3 * ((nfmax + 127) / 128));
    }
    // the first iterate of a pair launch whose second iteration carries the
    // check (the final u when it passes)
    if (op->kind == kAniso && !op->huber) {
        A((void **)&ws->an_img, (size_t)B * sizeof(AnImage));
        A((void **)&ws->an_st, (size_t)B * sizeof(AnState));
        A(&ws->an_scratch, img);
        A((void **)&ws->an_flag, (size_t)B * (size_t)N);
        A((void **)&ws->an_parent, (size_t)B * (size_t)N * sizeof(int));
        A((void **)&ws->an_cnt, (size_t)B * (size_t)N * sizeof(int));
        A((void **)&ws->an_sum, (size_t)B * (size_t)N * sizeof(unsigned long long));
        A(&ws->an_ys, img);
        A(&ws->an_segv, img);
        A((void **)&ws->an_segk, (size_t)B * (size_t)N * sizeof(int));
        if (!op->spatial.empty()) A(&ws->an_wt, op->spatial.size() * T);
    }
    if (ws->keep) {
        const size_t bn = (size_t)B * (size_t)N, kk = (size_t)g.k;
        A((void **)&ws->v_flat, bn);
        if (op->kind == kAniso) {
            A((void **)&ws->v_code, bn);
            A((void **)&ws->v_side, bn);
        }
        A((void **)&ws->v_root, bn * sizeof(int));
        A((void **)&ws->v_cnt, bn * sizeof(int));
        A((void **)&ws->v_gz, kk * bn * sizeof(double));
        A((void **)&ws->v_h, kk * bn * sizeof(double));
        A((void **)&ws->v_vec, 7 * bn * sizeof(double));
        A((void **)&ws->v_acc, 2 * bn * sizeof(unsigned long long));
        static_assert(sizeof(VjpImage) == sizeof(AnVjpImage), "one per-image record of the kept point");
        A((void **)&ws->v_img, (size_t)B * sizeof(VjpImage));
        A((void **)&ws->v_cg, (size_t)B * sizeof(CgState));
        A((void **)&ws->v_ggam, (size_t)B * sizeof(double));
        A((void **)&ws->v_gw, (size_t)B * 3 * sizeof(double));
    }
    A((void **)&ws->img, (size_t)B * sizeof(IsoImage));
    A((void **)&ws->st, (size_t)B * sizeof(IsoState));
    A((void **)&ws->gammas, (size_t)B * sizeof(double));
    A((void **)&ws->part, (size_t)B * (size_t)ws->max_part * 2 * sizeof(double));
    A((void **)&ws->ticket, (size_t)B * sizeof(unsigned));
    A((void **)&ws->lmap, (size_t)B * sizeof(int));
    A((void **)&ws->lcnt, sizeof(int));
    A((void **)&ws->live, 16);
    A((void **)&ws->err, 16);
    auto H = [&](void **p, size_t bytes) { host.add(p, bytes); };
    H((void **)&ws->h_live, 4 * sizeof(int));
    H((void **)&ws->h_img, (size_t)B * sizeof(IsoImage));
    H((void **)&ws->h_st, (size_t)B * sizeof(IsoState));
    H((void **)&ws->h_gam, (size_t)B * sizeof(double));
    if (ws->keep) {
        H((void **)&ws->h_vimg, (size_t)B * sizeof(VjpImage));
        H((void **)&ws->h_cg, (size_t)B * sizeof(CgState));
        H((void **)&ws->h_ggam, (size_t)B * sizeof(double));
        H((void **)&ws->h_gw, (size_t)B * 3 * sizeof(double));
    }
    if (op->kind == kAniso && !op->huber) {
        H((void **)&ws->h_an_img, (size_t)B * sizeof(AnImage));
        H((void **)&ws->h_an_st, (size_t)B * sizeof(AnState));
    }
    if (ws->host_mode) H(&ws->h_stage, img);
    // one pinned block and one device block from the pools (no device-wide
    // synchronisation); tickets and the error flag start at zero
    ws->host_bytes = host.total;
    ws->host_block = pinned_take(host.total);
    if (!ws->host_block) s = FP_ENOMEM;
    if (s == FP_OK) {
        host.place(ws->host_block);
        std::memset(ws->host_block, 0, host.total);
        void *base = nullptr;
        const cudaError_t e = pool_alloc(device, dev.total, &base, [&](cudaStream_t ps) {
            dev.place(base);
            cudaError_t r = cudaMemsetAsync(ws->ticket, 0, (size_t)B * sizeof(unsigned), ps);
            if (r == cudaSuccess) r = cudaMemsetAsync(ws->err, 0, 16, ps);
            if (r == cudaSuccess && !spatial_h.empty())
                r = cudaMemcpyAsync(ws->spatial, spatial_h.data(), spatial_h.size(), cudaMemcpyHostToDevice, ps);
            if (r == cudaSuccess && ws->an_wt && N > 0) {  // the edge weights of strided axes, fibre-major
                AnGeom ag{};
                ag.k = g.k;
                for (int a = 0; a < 3; ++a) ag.L[a] = a < g.k ? g.L[a] : 1;
                ag.S[g.k - 1] = 1;
                for (int a = g.k - 2; a >= 0; --a) ag.S[a] = ag.S[a + 1] * ag.L[a + 1];
                for (int a = g.k; a < 3; ++a) ag.S[a] = 1;
                ag.N = N;
                ag.B = B;
                r = aniso_weights_fm(x.dtype, ag, ws->spatial, ws->an_wt, ps);
            }
            return r;
        });
        ws->dev_block = base;
        if (e != cudaSuccess) s = e == cudaErrorMemoryAllocation ? FP_ENOMEM : FP_EDEVICE;
    }
    for (int i = 0; i < 2 && s == FP_OK; ++i)
        if (cudaEventCreateWithFlags(&ws->ev[i], cudaEventDisableTiming) != cudaSuccess) s = FP_EDEVICE;
    if (s != FP_OK) {
        cudaGetLastError();
        free_ws_memory(ws.get());
        return s;
    }
    ws->gaps.assign((size_t)B, 0.0);
    ws->zerrs.assign((size_t)B, 0.0);
    ws->iters.assign((size_t)B, 0);
    *out = ws.release();
    return FP_OK;
}

extern "C" {

FP_API fp_status fp_workspace_create(const fp_op *op, const fp_array *like, const fp_options *opt,
                                     fp_workspace **out) {
    return guard([&] {
        if (!out) return FP_EINVAL;
        *out = nullptr;
        if (!op || !like) return FP_EINVAL;
        const fp_options o = opt ? *opt : defaults();
        Arr x;
        if (fp_status s = to_arr(like, x)) return s;
        if (x.ndim < op->k) return FP_ESHAPE;
        if (x.numel() != 0)
            if (fp_status s = check_image(*op, x)) return s;
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            return FP_EDEVICE;
        }
        int device = 0;
        if (x.device == FP_DEVICE_CUDA) {
            device = x.data ? pointer_device(x.data) : -1;
            if (device < 0) {
                if (x.data) return FP_EINVAL;  // not device memory
                cudaGetDevice(&device);
            }
        } else {
            cudaGetDevice(&device);
        }
        return fpb_workspace_build(op, x, o, device, out);
    });
}

FP_API void fp_workspace_free(fp_workspace *ws) {
    if (!ws) return;
    free_ws_memory(ws);
    delete ws;
}

FP_API fp_status fp_workspace_set_stream(fp_workspace *ws, void *stream) {
    if (!ws) return FP_EINVAL;
    if (ws->host_mode) return FP_EINVAL;
    ws->stream = static_cast<cudaStream_t>(stream);
    return FP_OK;
}

FP_API fp_status fp_workspace_get_stream(const fp_workspace *ws, void **stream) {
    if (!ws || !stream) return FP_EINVAL;
    if (ws->host_mode) return FP_EINVAL;
    *stream = ws->stream;
    return FP_OK;
}

FP_API fp_status fp_workspace_set_warm(fp_workspace *ws, int on) {
    if (!ws) return FP_EINVAL;
    ws->warm = on != 0;
    return FP_OK;
}

FP_API fp_status fp_workspace_set_deriv_tol(fp_workspace *ws, double tol, int max_iter) {
    if (!ws) return FP_EINVAL;
    if (!(tol >= 0.0) || !std::isfinite(tol) || max_iter < 1) return FP_EPARAM;
    ws->deriv_tol = tol;
    ws->deriv_max_iter = max_iter;
    return FP_OK;
}

FP_API fp_status fp_workspace_deriv_info(const fp_workspace *ws, double *residual, int *iters) {
    if (!ws) return FP_EINVAL;
    if (residual) *residual = ws->deriv_residual;
    if (iters) *iters = ws->deriv_iters;
    return FP_OK;
}

FP_API fp_status fp_workspace_info(const fp_workspace *ws, fp_info *info) {
    if (!ws || !info) return FP_EINVAL;
    if (!ws->info_valid) return FP_EINVAL;
    *info = ws->info;
    return ws->info_status;
}

FP_API fp_status fp_workspace_image_info(const fp_workspace *ws, double *gaps, int *iters, double *zerrs,
                                         int64_t count) {
    if (!ws) return FP_EINVAL;
    if (!ws->info_valid) return FP_EINVAL;
    if (count != ws->g.B) return FP_ESHAPE;
    for (int64_t i = 0; i < count; ++i) {
        if (gaps) gaps[i] = ws->gaps[(size_t)i];
        if (iters) iters[i] = ws->iters[(size_t)i];
        if (zerrs) zerrs[i] = ws->zerrs[(size_t)i];
    }
    return FP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The dual: get, set (src/api/api.cpp dual_impl; fastprox.h:415-428)
// ---------------------------------------------------------------------------

namespace {

fp_status dual_io(fp_workspace *ws, const fp_array *arr, bool set) {
    if (!ws || !arr) return FP_EINVAL;
    Arr a;
    if (fp_status s = to_arr(arr, a)) return s;
    // shape (k, *x.shape)
    if (a.ndim != ws->ndim + 1 || a.shape[0] != ws->g.k) return FP_ESHAPE;
    for (int d = 0; d < ws->ndim; ++d)
        if (a.shape[d + 1] != ws->shape[d]) return FP_ESHAPE;
    if (!set && !ws->dual_valid) return FP_EINVAL;
    const int64_t n = a.numel();
    if (n == 0) {
        if (set) {
            ws->seeded = true;
            ws->dual_valid = true;
        }
        return FP_OK;
    }
    DeviceScope dsc(ws->device);
    const size_t T = ws->dtype == FP_F32 ? 4 : 8;
    int64_t cst[FP_MAX_NDIM];
    {
        int64_t s = 1;
        for (int d = a.ndim - 1; d >= 0; --d) {
            cst[d] = s;
            s *= a.shape[d];
        }
    }
    cudaStream_t st = ws->stream;
    if (a.device == FP_DEVICE_CUDA) {
        if (pointer_device(a.data) != ws->device) return FP_EINVAL;
        if (set) {
            // Inf entries are rejected, NaN entries stored as 0.
            std::vector<char> hostcopy((size_t)n * a.itemsize());
            cudaError_t e = cudaSuccess;
            if (a.contiguous()) {
                e = cudaMemcpyAsync(ws->dual, a.data, (size_t)n * T, cudaMemcpyDeviceToDevice, st);
                if (a.dtype != ws->dtype) {
                    e = strided_copy(a.data, a.dtype, a.shape, a.strides, a.ndim, ws->dual, ws->dtype, cst, st);
                }
            } else {
                e = strided_copy(a.data, a.dtype, a.shape, a.strides, a.ndim, ws->dual, ws->dtype, cst, st);
            }
            if (e != cudaSuccess) return cuda_status(e);
            // validate on the host
            std::vector<char> h((size_t)n * T);
            if (cudaMemcpyAsync(h.data(), ws->dual, h.size(), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                return FP_EDEVICE;
            bool bad = false;
            for (int64_t i = 0; i < n; ++i) {
                double v = T == 4 ? (double)reinterpret_cast<float *>(h.data())[i] : reinterpret_cast<double *>(h.data())[i];
                if (std::isinf(v)) bad = true;
                if (std::isnan(v)) {
                    if (T == 4) reinterpret_cast<float *>(h.data())[i] = 0.0f;
                    else reinterpret_cast<double *>(h.data())[i] = 0.0;
                }
            }
            if (bad) return FP_EINVAL;
            if (cudaMemcpyAsync(ws->dual, h.data(), h.size(), cudaMemcpyHostToDevice, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                return FP_EDEVICE;
            ws->seeded = true;
            ws->dual_valid = true;
            return FP_OK;
        }
        cudaError_t e = strided_copy(ws->dual, ws->dtype, a.shape, cst, a.ndim, a.data, a.dtype, a.strides, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        return cuda_status(e);
    }
    // host array
    std::vector<char> h((size_t)n * T);
    if (set) {
        std::vector<int64_t> idx((size_t)a.ndim, 0);
        bool bad = false;
        for (int64_t i = 0; i < n; ++i) {
            int64_t off = 0;
            for (int d = 0; d < a.ndim; ++d) off += idx[(size_t)d] * a.strides[d];
            const char *p = a.data + off * (int64_t)a.itemsize();
            double v = a.dtype == FP_F32 ? (double)*reinterpret_cast<const float *>(p) : *reinterpret_cast<const double *>(p);
            if (std::isinf(v)) bad = true;
            if (std::isnan(v)) v = 0.0;
            if (T == 4) reinterpret_cast<float *>(h.data())[i] = (float)v;
            else reinterpret_cast<double *>(h.data())[i] = v;
            for (int d = a.ndim - 1; d >= 0; --d) {
                if (++idx[(size_t)d] < a.shape[d]) break;
                idx[(size_t)d] = 0;
            }
        }
        if (bad) return FP_EINVAL;
        if (cudaMemcpyAsync(ws->dual, h.data(), h.size(), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return FP_EDEVICE;
        ws->seeded = true;
        ws->dual_valid = true;
        return FP_OK;
    }
    if (cudaMemcpyAsync(h.data(), ws->dual, h.size(), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return FP_EDEVICE;
    std::vector<int64_t> idx((size_t)a.ndim, 0);
    for (int64_t i = 0; i < n; ++i) {
        int64_t off = 0;
        for (int d = 0; d < a.ndim; ++d) off += idx[(size_t)d] * a.strides[d];
        char *p = a.data + off * (int64_t)a.itemsize();
        const double v = T == 4 ? (double)reinterpret_cast<float *>(h.data())[i] : reinterpret_cast<double *>(h.data())[i];
        if (a.dtype == FP_F32) *reinterpret_cast<float *>(p) = (float)v;
        else *reinterpret_cast<double *>(p) = v;
        for (int d = a.ndim - 1; d >= 0; --d) {
            if (++idx[(size_t)d] < a.shape[d]) break;
            idx[(size_t)d] = 0;
        }
    }
    return FP_OK;
}

}  // namespace

extern "C" {

FP_API fp_status fp_workspace_get_dual(const fp_workspace *ws, fp_array *out) {
    return guard([&] { return dual_io(const_cast<fp_workspace *>(ws), out, false); });
}

FP_API fp_status fp_workspace_set_dual(fp_workspace *ws, const fp_array *dual) {
    return guard([&] { return dual_io(ws, dual, true); });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// prox
// ---------------------------------------------------------------------------

namespace {

// Per-image certified relative error of the returned z (driver.hpp:1187-1237):
// r + round (u (1 + r) + a / |x|), r = sqrt(2 gap) / |x|, at the solved scale.
double certified_error(double gap_s, double dd_s, int64_t N, int e, int dtype, int round) {
    if (std::isnan(gap_s)) return gap_s;
    if (!(dd_s > 0.0)) return 0.0;
    const double u = 0.5 * (dtype == FP_F32 ? (double)std::numeric_limits<float>::epsilon()
                                            : std::numeric_limits<double>::epsilon());
    const double eta = 0.5 * (dtype == FP_F32 ? (double)std::numeric_limits<float>::denorm_min()
                                              : std::numeric_limits<double>::denorm_min());
    const double n = std::sqrt(dd_s);
    const double r = std::sqrt(2.0 * std::max(gap_s, 0.0)) / n;
    const double a = std::ldexp(eta, -e) * std::sqrt((double)N) / n;
    return r + round * (u * (1.0 + r) + a);
}

fp_status run_iso(fp_workspace *ws, const fp_op *op, const void *xsrc, void *zdst, double tol, int max_iter,
                  bool warm) {
    const Geometry &g = ws->g;
    cudaStream_t s = ws->stream;
    IsoCall c{};
    // Active axes (tv_iso.cpp:350-358) for a positive step
    double wmax_all = 0.0;
    for (int a = 0; a < g.k; ++a)
        if (g.L[a] > 1) wmax_all = std::max(wmax_all, op->w[a]);
    double wa[3] = {0.0, 0.0, 0.0};
    int na = 0, act = -1;
    for (int a = 0; a < g.k; ++a)
        if (op->w[a] > 0.0 && g.L[a] > 1 && op->w[a] >= 1e-100 * wmax_all) {
            wa[a] = op->w[a];
            ++na;
            act = a;
        }
    c.na = na;
    c.act_axis = act < 0 ? 0 : act;
    c.w_act = act < 0 ? 1.0 : op->w[act];
    double wmax = 0.0;
    for (int a = 0; a < g.k; ++a) wmax = std::max(wmax, wa[a]);
    c.wmax = wmax > 0.0 ? wmax : 1.0;
    double whmin = 1.0, L2 = 0.0;
    for (int a = 0; a < 3; ++a) {
        c.wh[a] = (a < g.k && wa[a] != 0.0) ? wa[a] / c.wmax : 0.0;
        if (a < g.k && wa[a] != 0.0) whmin = std::min(whmin, c.wh[a]);
        L2 += 4.0 * c.wh[a] * c.wh[a];
    }
    c.whmin = whmin;
    c.tau = L2 > 0.0 ? 1.0 / L2 : 0.0;
    c.tol = tol;
    c.max_iter = max_iter;
    c.has_alpha = op->spatial.empty() ? 0 : 1;
    c.alpha_stride = 0;
    c.alpha_max = op->smax;
    c.step_scale = std::max({op->w[0], op->w[1], op->w[2]}) * (op->spatial.empty() ? 1.0 : op->smax);
    c.huber = op->huber ? (op->kind == kIso ? 1 : 2) : 0;
    c.delta = op->delta;

    IsoBuffers bf;
    bf.d = ws->d;
    for (int i = 0; i < 2; ++i) {
        bf.U[i] = ws->U[i];
        bf.V[i] = ws->V[i];
    }
    bf.dual = ws->dual;
    bf.alpha = ws->spatial;
    bf.img = ws->img;
    bf.st = ws->st;
    bf.gammas = ws->gammas;
    bf.part = ws->part;
    bf.ticket = ws->ticket;
    bf.live = ws->live;
    bf.err = ws->err;
    bf.max_part = ws->max_part;

    cudaError_t e = cudaMemsetAsync(ws->live, 0, sizeof(int), s);
    if (e == cudaSuccess) e = iso_setup(ws->dtype, g, c, bf, xsrc, warm ? 1 : 0, 0, s);
    if (e != cudaSuccess) return cuda_status(e);
    // The iteration: chunks of launches, each followed by a read of the live
    // count; two chunks in flight so the device never waits for the host.
    // Once fewer images are live than the launches cover, the launches cover
    // a list of the live ones (images only retire, so a list built after the
    // count was read holds every image still live): the tail of a batch, where
    // a few slow images remain, launches only their blocks.
    // Iterations 1 and 2 mod 4 (no check in either), and 3 and 4 mod 4 (the
    // second with the check) run as one launch each where the lean 2D step
    // applies (iso_pair_ok).
    const int chunk = ws->chunk > 0 ? ws->chunk : 8;
    const bool pairs = iso_pair_ok(g, ws->shape_, ws->max_part);
    const bool quads = !c.huber && iso_quad_ok(ws->dtype, g, ws->max_part);
    int par = 0, slot = 0, inflight = 0;
    int64_t launched = 0, steps = 0, lists = 0, nimg = g.B;
    const int64_t cap = (int64_t)max_iter + 1 + 2 * chunk;
    // step-launch timing: an event pair around each launch, up to kTimed launches
    constexpr size_t kTimed = 4096;
    std::vector<int> tkind;
    for (int k = 0; k < 4; ++k) {
        ws->tms[k] = 0.0;
        ws->tcount[k] = 0;
    }
    bool done = false;
    while (!done) {
        for (int j = 0; j < chunk; ++j) {
            int pv = quads ? iso_quad_at(launched, max_iter) : -1;
            if (pv < 0 && pairs) pv = iso_pair_at(launched, max_iter);
            const bool timed = ws->time_steps && tkind.size() < kTimed;
            if (timed) {
                while (ws->tev.size() < 2 * (tkind.size() + 1)) {
                    cudaEvent_t ev = nullptr;
                    if ((e = cudaEventCreate(&ev)) != cudaSuccess) return cuda_status(e);
                    ws->tev.push_back(ev);
                }
                if ((e = cudaEventRecord(ws->tev[2 * tkind.size()], s)) != cudaSuccess) return cuda_status(e);
            }
            e = iso_step(ws->dtype, g, c, bf, ws->shape_, par, pv >= 0 ? pv : iso_variant(launched, max_iter, warm),
                         nimg, s);
            if (e != cudaSuccess) return cuda_status(e);
            if (timed) {
                if ((e = cudaEventRecord(ws->tev[2 * tkind.size() + 1], s)) != cudaSuccess) return cuda_status(e);
                tkind.push_back(pv == kVariantQuad ? 3 : pv == kVariantPairGap ? 2 : (pv == kVariantPair ? 1 : 0));
            }
            par ^= 1;
            launched += pv == kVariantQuad ? 4 : pv >= 0 ? 2 : 1;
            ++steps;
        }
        e = cudaMemcpyAsync(ws->h_live + slot, ws->live, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaEventRecord(ws->ev[slot], s);
        if (e != cudaSuccess) return cuda_status(e);
        slot ^= 1;
        ++inflight;
        if (inflight == 2) {
            e = cudaEventSynchronize(ws->ev[slot]);
            if (e != cudaSuccess) return cuda_status(e);
            --inflight;
            const int live = ws->h_live[slot];
            if (live == 0) {
                done = true;
            } else if (live < nimg) {
                e = iso_live_list(ws->st, g.B, ws->lmap, ws->lcnt, s);
                if (e != cudaSuccess) return cuda_status(e);
                bf.lmap = ws->lmap;
                bf.lcnt = ws->lcnt;
                nimg = live;
                ++lists;
            }
        }
        if (launched >= cap) done = true;
    }
    ws->launches = steps;
    ws->kernel_launches += steps + lists + 3 + (warm ? 1 : 0) + 1 + ((c.na == 1 && !c.has_alpha) ? 1 : 0);
    if (!tkind.empty()) {
        if ((e = cudaEventSynchronize(ws->tev[2 * tkind.size() - 1])) != cudaSuccess) return cuda_status(e);
        for (size_t k = 0; k < tkind.size(); ++k) {
            float ms = 0.0f;
            if ((e = cudaEventElapsedTime(&ms, ws->tev[2 * k], ws->tev[2 * k + 1])) != cudaSuccess)
                return cuda_status(e);
            ws->tms[tkind[k]] += ms;
            ws->tcount[tkind[k]] += 1;
        }
    }
    if (pairs || quads) {
        e = iso_redo(ws->dtype, g, c, bf, s, quads);
        ws->kernel_launches += quads ? 3 : 2;
    }
    if (e == cudaSuccess) e = iso_finalize(ws->dtype, g, c, bf, zdst, s);
    return cuda_status(e);
}

// Anisotropic rounds per captured graph, and the solves that use graphs: a
// round is about 15 launches, most of which exit at once, so a small solve is
// bound by launch latency (a 64 x 64 image took 150 us a round in plain
// launches). FASTPROX_B200_AN_GRAPHS=0 keeps plain launches.
constexpr int kAnChunk = 4;
constexpr int64_t kAnGraphPixels = int64_t(1) << 22;

bool an_graphs_enabled() {
    static const bool on = [] {
        const char *v = std::getenv("FASTPROX_B200_AN_GRAPHS");
        return !(v && v[0] == '0' && v[1] == 0);
    }();
    return on;
}

bool same_call(const AnCall &a, const AnCall &b) {
    return a.w[0] == b.w[0] && a.w[1] == b.w[1] && a.w[2] == b.w[2] && a.tol == b.tol && a.max_iter == b.max_iter &&
           a.step_scale == b.step_scale && a.has_beta == b.has_beta && a.beta_max == b.beta_max && a.N == b.N &&
           a.has_adbpg == b.has_adbpg && a.has_fdpg3 == b.has_fdpg3 && a.warm == b.warm;
}

// kAnChunk rounds as one graph launch on s, captured on a private stream when
// the workspace holds none for these arguments. False: capture failed (the
// caller launches rounds itself from then on).
bool an_graph_rounds(fp_workspace *ws, const AnGeom &g, const AnCall &c, const AnBuffers &bf, int64_t nimg,
                     cudaStream_t s, int64_t *launches, cudaError_t *err) {
    if (!(ws->an_graph && ws->an_graph_nimg == nimg && ws->an_graph_lmap == bf.lmap && same_call(ws->an_graph_c, c))) {
        if (ws->an_graph) cudaGraphExecDestroy(ws->an_graph);
        ws->an_graph = nullptr;
        cudaStream_t cap = nullptr;
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        cudaGraph_t graph = nullptr;
        int64_t nl = 0;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            for (int r = 0; r < kAnChunk && e == cudaSuccess; ++r) e = aniso_round(ws->dtype, g, c, bf, nimg, cap, &nl);
            const cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
            if (e == cudaSuccess) e = e2;
        }
        cudaStreamDestroy(cap);
        cudaGraphExec_t exec = nullptr;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        ws->an_graph = exec;
        ws->an_graph_c = c;
        ws->an_graph_nimg = nimg;
        ws->an_graph_lmap = bf.lmap;
        ws->an_graph_launches = nl;
    }
    *err = cudaGraphLaunch(ws->an_graph, s);
    *launches += ws->an_graph_launches;
    return true;
}

fp_status run_aniso(fp_workspace *ws, const fp_op *op, const void *xsrc, void *zdst, double tol, int max_iter,
                    bool warm) {
    const Geometry &g0 = ws->g;
    cudaStream_t s = ws->stream;
    const size_t T = ws->dtype == FP_F32 ? 4 : 8;
    AnGeom g{};
    g.k = g0.k;
    for (int a = 0; a < 3; ++a) g.L[a] = g0.L[a];
    g.S[g.k - 1] = 1;
    for (int a = g.k - 2; a >= 0; --a) g.S[a] = g.S[a + 1] * g.L[a + 1];
    for (int a = g.k; a < 3; ++a) g.S[a] = 1;
    g.N = g0.N;
    g.B = g0.B;
    AnCall c{};
    int na = 0;
    for (int a = 0; a < 3; ++a) {
        c.w[a] = a < g.k ? op->w[a] : 0.0;
        if (a < g.k && op->w[a] > 0.0 && g.L[a] > 1) ++na;
    }
    c.tol = tol;
    c.max_iter = max_iter;
    c.has_beta = op->spatial.empty() ? 0 : 1;
    c.beta_max = op->spatial.empty() ? 1.0 : op->smax;
    c.step_scale = std::max({op->w[0], op->w[1], op->w[2]}) * (op->spatial.empty() ? 1.0 : op->smax);
    c.N = g.N;
    c.has_adbpg = na == 2;
    c.has_fdpg3 = na == 3;
    AnBuffers bf;
    const size_t bn = (size_t)g.B * (size_t)g.N;
    bf.d = ws->d;
    bf.y = ws->U[0];
    bf.wv = ws->V[0];
    bf.z = ws->U[1];
    bf.zp = static_cast<char *>(ws->U[1]) + bn * T;
    bf.u = ws->V[1];
    bf.scratch = ws->an_scratch;
    bf.dual = ws->dual;
    bf.beta = ws->spatial;
    bf.flag = ws->an_flag;
    bf.parent = ws->an_parent;
    bf.sum = ws->an_sum;
    bf.cnt = ws->an_cnt;
    bf.ys = ws->an_ys;
    bf.segv = ws->an_segv;
    bf.segk = ws->an_segk;
    bf.wt = ws->an_wt;
    bf.img = ws->an_img;
    bf.st = ws->an_st;
    bf.gammas = ws->gammas;
    bf.part = ws->part;
    bf.ticket = ws->ticket;
    bf.live = ws->live;
    bf.err = ws->err;
    bf.max_part = ws->max_part;
    cudaError_t e = cudaMemsetAsync(ws->live, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws->U[0], 0, (size_t)g.k * bn * T, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws->V[0], 0, (size_t)g.k * bn * T, s);
    if (e == cudaSuccess) e = aniso_setup(ws->dtype, g, c, bf, xsrc, s);
    c.warm = warm && (c.has_adbpg || c.has_fdpg3) ? 1 : 0;
    if (e == cudaSuccess && c.warm) e = aniso_warm(ws->dtype, g, c, bf, s);
    if (e != cudaSuccess) return cuda_status(e);
    int64_t launches = 5;
    aniso_prepare(ws->dtype);
    // rounds of launches (an iteration each, with its check, polish and
    // retirement), the live count read back behind two rounds in flight
    // (over a list of the live images once fewer are live, as in run_iso);
    // after the first, small solves replay rounds in captured chunks
    int slot = 0, inflight = 0;
    int64_t rounds = 0, nimg = g.B;
    const int64_t cap = (int64_t)max_iter + 4;
    bool done = false;
    bool graphs = an_graphs_enabled() && g.N * g.B <= kAnGraphPixels;
    while (!done) {
        if (graphs && rounds > 0 && an_graph_rounds(ws, g, c, bf, nimg, s, &launches, &e)) {
            rounds += kAnChunk;
        } else {
            if (rounds > 0) graphs = false;
            e = aniso_round(ws->dtype, g, c, bf, nimg, s, &launches);
            ++rounds;
        }
        if (e != cudaSuccess) return cuda_status(e);
        e = cudaMemcpyAsync(ws->h_live + slot, ws->live, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaEventRecord(ws->ev[slot], s);
        if (e != cudaSuccess) return cuda_status(e);
        slot ^= 1;
        ++inflight;
        if (inflight == 2) {
            e = cudaEventSynchronize(ws->ev[slot]);
            if (e != cudaSuccess) return cuda_status(e);
            --inflight;
            const int live = ws->h_live[slot];
            if (live == 0) {
                done = true;
            } else if (live < nimg) {
                e = aniso_live_list(ws->an_st, g.B, ws->lmap, ws->lcnt, s);
                if (e != cudaSuccess) return cuda_status(e);
                bf.lmap = ws->lmap;
                bf.lcnt = ws->lcnt;
                nimg = live;
                ++launches;
            }
        }
        if (rounds >= cap) done = true;
    }
    ws->launches = rounds;
    ws->kernel_launches += launches + 1;
    e = aniso_output(ws->dtype, g, bf, zdst, s);
    return cuda_status(e);
}

fp_status copy_or_fill(fp_workspace *ws, const Arr *src, const Arr &dst, double fill, void *scratch);

fp_status prox_impl(const fp_op *op, double step, const fp_array *xa, fp_array *oa, const fp_options *opt,
                    fp_workspace *ws, fp_info *info, bool conj, const fp_array *sa) {
    if (!op || !xa || !oa) return FP_EINVAL;
    if (!std::isfinite(step) || step < 0) return FP_EPARAM;
    const fp_options o = opt ? *opt : defaults();
    if (o.tie != 0 && o.tie != 1) return FP_EINVAL;
    Arr x, out;
    if (fp_status s = to_arr(xa, x)) return s;
    if (fp_status s = to_arr(oa, out)) return s;
    if (x.dtype != out.dtype) return FP_EDTYPE;
    if (!same_shape(x, out)) return FP_ESHAPE;
    if (x.device != out.device) return FP_EINVAL;
    if (fp_status s = check_output(&x, out)) return s;
    const bool keep = o.keep_structure != 0;
    if (keep && !ws) return FP_EINVAL;
    if (ws) {
        if (ws->op != op || ws->dtype != x.dtype || ws->ndim != x.ndim) return FP_EINVAL;
        for (int d = 0; d < x.ndim; ++d)
            if (ws->shape[d] != x.shape[d]) return FP_ESHAPE;
        if (keep && !ws->keep) return FP_EINVAL;
        if (ws->host_mode != (x.device == FP_DEVICE_CPU)) return FP_EINVAL;
    }
    if (info) {
        info->gap = 0.0;
        info->iters = 0;
        info->ties = 0;
    }
    const int k = op->k;
    if (x.ndim < k) return FP_ESHAPE;
    if (!(o.tol >= 0.0) || !std::isfinite(o.tol) || o.max_iter < 1) return FP_EPARAM;
    const double step_scale = std::max({op->w[0], op->w[1], op->w[2]}) * (op->spatial.empty() ? 1.0 : op->smax);
    const bool identity = conj && step == 0.0;
    const double gamma = conj ? 1.0 : step;  // TV is positively homogeneous (api.cpp:463-469)
    Arr st;
    Geometry g0;
    if (fp_status s = image_geometry(*op, x, g0)) return s;
    // The steps per image, read into the workspace's pinned buffer (a call
    // with a workspace allocates nothing on the host either), or into a local
    // one when the call builds its own workspace.
    std::vector<double> local_steps;
    double *host_steps = nullptr;
    bool device_steps = false;
    if (sa) {
        if (fp_status s = to_arr(sa, st)) return s;
        if (sa->ndim != x.ndim - k) return FP_ESHAPE;
        for (int d = 0; d < sa->ndim; ++d)
            if (st.shape[d] != x.shape[d]) return FP_ESHAPE;
        if (fp_status s = check_output(&st, out)) return s;
        // every step checked before any work
        const int64_t B = g0.B;
        if (ws) {
            host_steps = ws->h_gam;
        } else {
            local_steps.resize((size_t)std::max<int64_t>(B, 1));
            host_steps = local_steps.data();
        }
        if (st.device == FP_DEVICE_CPU) {
            int64_t idx[FP_MAX_NDIM] = {0};
            for (int64_t i = 0; i < B; ++i) {
                int64_t off = 0;
                for (int d = 0; d < sa->ndim; ++d) off += idx[d] * st.strides[d];
                const char *p = st.data + off * (int64_t)st.itemsize();
                host_steps[i] = st.dtype == FP_F32 ? (double)*reinterpret_cast<const float *>(p)
                                                   : *reinterpret_cast<const double *>(p);
                for (int d = sa->ndim - 1; d >= 0; --d) {
                    if (++idx[d] < st.shape[d]) break;
                    idx[d] = 0;
                }
            }
        } else {
            device_steps = true;  // read into the workspace below, checked before any work
        }
        if (!device_steps)
            for (int64_t i = 0; i < B; ++i) {
                const double v = host_steps[i];
                if (!std::isfinite(v) || v < 0) return FP_EPARAM;
                if (step_scale > 0.0 && !(v * step_scale <= kMaxScaledStep)) return FP_EPARAM;
            }
    } else if (!identity && step_scale > 0.0 && !(gamma * step_scale <= kMaxScaledStep)) {
        return FP_EPARAM;
    }
    if (x.numel() != 0)
        if (fp_status s = check_image(*op, x)) return s;
    if (ws) {
        ws->valid = false;
        ws->info_valid = false;
        ws->struct_valid = false;
        ws->identity = false;
        ws->branch_on = false;  // an override belongs to the point it was set for
        ws->conj = conj;
    }
    if (x.numel() == 0) {
        if (ws) {
            ws->dual_valid = true;
            ws->info = fp_info{0.0, 0, 0};
            ws->info_status = FP_OK;
            ws->info_valid = true;
        }
        return FP_OK;
    }
    // The device: the workspace's, or that of the arrays.
    std::unique_ptr<fp_workspace, void (*)(fp_workspace *)> local(nullptr, fp_workspace_free);
    if (!ws) {
        int device = 0;
        if (x.device == FP_DEVICE_CUDA) {
            device = pointer_device(x.data);
            if (device < 0) return FP_EINVAL;
        } else {
            int n = 0;
            if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
                cudaGetLastError();
                return FP_EDEVICE;
            }
            cudaGetDevice(&device);
        }
        fp_workspace *w = nullptr;
        if (fp_status s = fpb_workspace_build(op, x, o, device, &w)) return s;
        local.reset(w);
        ws = w;
    }
    DeviceScope dsc(ws->device);
    if (x.device == FP_DEVICE_CUDA) {
        if (pointer_device(x.data) != ws->device || pointer_device(out.data) != ws->device) return FP_EINVAL;
    }
    if (identity) {
        // sigma = 0 in the conjugate: y itself, and with keep the identity's
        // derivatives (api.cpp:529-534)
        if (fp_status st = copy_or_fill(ws, &x, out, 0.0, nullptr)) return st;
        std::fill(ws->gaps.begin(), ws->gaps.end(), 0.0);
        std::fill(ws->zerrs.begin(), ws->zerrs.end(), 0.0);
        std::fill(ws->iters.begin(), ws->iters.end(), 0);
        ws->seeded = false;
        if (keep) {
            ws->valid = true;
            ws->identity = true;
        }
        ws->info = fp_info{0.0, 0, 0};
        ws->info_status = FP_OK;
        ws->info_valid = true;
        return FP_OK;
    }
    if (device_steps) {
        // the steps into the workspace (as doubles), read back and checked
        if (pointer_device(st.data) != ws->device) return FP_EINVAL;
        int64_t one[FP_MAX_NDIM];
        int64_t sz = 1;
        for (int d = sa->ndim - 1; d >= 0; --d) {
            one[d] = sz;
            sz *= st.shape[d];
        }
        cudaError_t e0 = strided_copy(st.data, st.dtype, st.shape, st.strides, std::max(1, sa->ndim), ws->gammas,
                                      FP_F64, one, ws->stream);
        if (e0 == cudaSuccess)
            e0 = cudaMemcpyAsync(ws->h_gam, ws->gammas, (size_t)ws->g.B * sizeof(double), cudaMemcpyDeviceToHost,
                                 ws->stream);
        if (e0 == cudaSuccess) e0 = cudaStreamSynchronize(ws->stream);
        if (e0 != cudaSuccess) return cuda_status(e0);
        for (int64_t i = 0; i < ws->g.B; ++i) {
            const double v = ws->h_gam[i];
            if (!std::isfinite(v) || v < 0) return FP_EPARAM;
            if (step_scale > 0.0 && !(v * step_scale <= kMaxScaledStep)) return FP_EPARAM;
        }
    }
    cudaStream_t s = ws->stream;
    const Geometry &g = ws->g;
    const size_t T = x.itemsize();
    const int64_t total = g.B * g.N;
    int64_t cst[FP_MAX_NDIM];
    {
        int64_t sz = 1;
        for (int d = x.ndim - 1; d >= 0; --d) {
            cst[d] = sz;
            sz *= x.shape[d];
        }
    }
    ws->kernel_launches = 1;  // the steps fill (or strided copies, counted below)
    cudaError_t e = cudaSuccess;
    // Stage x: the kernels read a contiguous batch. The conjugate keeps y
    // in the staging buffer for out = y - z.
    const void *xsrc = nullptr;
    const void *ysave = nullptr;
    if (ws->host_mode) {
        if (x.contiguous() && host_pinned(x.data)) {
            e = cudaMemcpyAsync(ws->d, x.data, (size_t)total * T, cudaMemcpyHostToDevice, s);
        } else {
            // pack through the pinned staging buffer
            if (cudaStreamSynchronize(s) != cudaSuccess) return FP_EDEVICE;
            int64_t idx[FP_MAX_NDIM] = {0};
            char *hs = static_cast<char *>(ws->h_stage);
            for (int64_t i = 0; i < total; ++i) {
                int64_t off = 0;
                for (int d = 0; d < x.ndim; ++d) off += idx[d] * x.strides[d];
                std::memcpy(hs + i * (int64_t)T, x.data + off * (int64_t)T, T);
                for (int d = x.ndim - 1; d >= 0; --d) {
                    if (++idx[d] < x.shape[d]) break;
                    idx[d] = 0;
                }
            }
            e = cudaMemcpyAsync(ws->d, hs, (size_t)total * T, cudaMemcpyHostToDevice, s);
        }
        xsrc = ws->d;
        if (conj && e == cudaSuccess) {
            e = cudaMemcpyAsync(ws->stage, ws->d, (size_t)total * T, cudaMemcpyDeviceToDevice, s);
            ysave = ws->stage;
        }
    } else if (x.contiguous()) {
        xsrc = x.data;
        if (conj) {
            e = cudaMemcpyAsync(ws->stage, x.data, (size_t)total * T, cudaMemcpyDeviceToDevice, s);
            ysave = ws->stage;
        }
    } else {
        void *dst = conj ? ws->stage : ws->d;
        e = strided_copy(x.data, x.dtype, x.shape, x.strides, x.ndim, dst, x.dtype, cst, s);
        xsrc = dst;
        if (conj) ysave = dst;
    }
    if (e != cudaSuccess) return cuda_status(e);
    // Steps per image
    if (sa && !device_steps) {
        if (host_steps != ws->h_gam) std::memcpy(ws->h_gam, host_steps, (size_t)g.B * sizeof(double));
        e = cudaMemcpyAsync(ws->gammas, ws->h_gam, (size_t)g.B * sizeof(double), cudaMemcpyHostToDevice, s);
    } else if (!sa) {
        e = fill_double(ws->gammas, identity ? 0.0 : gamma, g.B, s);
    }
    if (e != cudaSuccess) return cuda_status(e);
    const bool warm = ws->dual_valid && (ws->warm || ws->seeded);
    // z: straight into a contiguous device out, else a device buffer free
    // at the end of the solve (stage, or V[1] when stage holds y)
    const bool direct_out = !ws->host_mode && out.contiguous();
    void *zdst = direct_out ? out.data : (conj ? ws->V[1] : ws->stage);
    if (op->kind == kIso || op->huber) {  // Huber-smoothed TV, either form, runs in the isotropic engine
        if (fp_status st2 = run_iso(ws, op, xsrc, zdst, o.tol, o.max_iter, warm)) return st2;
    } else {
        if (fp_status st2 = run_aniso(ws, op, xsrc, zdst, o.tol, o.max_iter, warm)) return st2;
    }
    if (conj) {
        e = conj_finish(ws->dtype, ysave, zdst, total, s);
        if (e != cudaSuccess) return cuda_status(e);
    }
    // Results back to the host
    if (op->kind == kIso || op->huber) {
        e = cudaMemcpyAsync(ws->h_img, ws->img, (size_t)g.B * sizeof(IsoImage), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ws->h_st, ws->st, (size_t)g.B * sizeof(IsoState), cudaMemcpyDeviceToHost, s);
    } else {
        e = cudaMemcpyAsync(ws->h_an_img, ws->an_img, (size_t)g.B * sizeof(AnImage), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ws->h_an_st, ws->an_st, (size_t)g.B * sizeof(AnState), cudaMemcpyDeviceToHost, s);
    }
    if (e != cudaSuccess) return cuda_status(e);
    if (!direct_out) {
        if (ws->host_mode) {
            if (out.contiguous() && host_pinned(out.data)) {
                e = cudaMemcpyAsync(out.data, zdst, (size_t)total * T, cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            } else {
                e = cudaMemcpyAsync(ws->h_stage, zdst, (size_t)total * T, cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e == cudaSuccess) {
                    int64_t idx[FP_MAX_NDIM] = {0};
                    const char *hs = static_cast<const char *>(ws->h_stage);
                    for (int64_t i = 0; i < total; ++i) {
                        int64_t off = 0;
                        for (int d = 0; d < out.ndim; ++d) off += idx[d] * out.strides[d];
                        std::memcpy(out.data + off * (int64_t)T, hs + i * (int64_t)T, T);
                        for (int d = out.ndim - 1; d >= 0; --d) {
                            if (++idx[d] < out.shape[d]) break;
                            idx[d] = 0;
                        }
                    }
                }
            }
        } else {
            e = strided_copy(zdst, out.dtype, out.shape, cst, out.ndim, out.data, out.dtype, out.strides, s);
        }
        if (e != cudaSuccess) return cuda_status(e);
    }
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    {
        // the device error flag (an internal consistency check), read on the stream
        e = cudaMemcpyAsync(ws->h_live + 3, ws->err, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e);
        if (ws->h_live[3]) {
            ws->h_live[3] = 0;
            cudaMemsetAsync(ws->err, 0, sizeof(int), s);
            cudaStreamSynchronize(s);
            return FP_EDEVICE;
        }
    }
    // Per-image results (driver.hpp:1303-1341)
    bool inf = false, notconv = false;
    double gsum = 0.0;
    int imax = 0;
    for (int64_t b = 0; b < g.B; ++b) {
        if (op->kind == kAniso && !op->huber) {
            const AnImage &im = ws->h_an_img[b];
            const AnState &sst = ws->h_an_st[b];
            double gap = 0.0, gap_s = 0.0;
            int it = 0;
            if (im.mode == kAnInf) {
                inf = true;
            } else if (im.mode == kAnNan) {
                gap = gap_s = std::numeric_limits<double>::quiet_NaN();
            } else if (im.mode == kAnAdbpg || im.mode == kAnFdpg3) {
                gap_s = std::isnan(sst.gp) ? sst.gp : std::max(sst.gp, 0.0);
                gap = im.e ? std::ldexp(gap_s, 2 * im.e) : gap_s;
                it = sst.it;
                if (sst.status != kConverged) notconv = true;
            }
            ws->gaps[(size_t)b] = gap;
            ws->iters[(size_t)b] = it;
            ws->zerrs[(size_t)b] = certified_error(gap_s, im.dd, g.N, im.e, ws->dtype, conj ? 2 : 1);
            gsum += gap;
            imax = std::max(imax, it);
            continue;
        }
        const IsoImage &im = ws->h_img[b];
        const IsoState &sst = ws->h_st[b];
        double gap = 0.0, gap_s = 0.0;
        int it = 0;
        if (im.mode == kModeInf) {
            inf = true;
        } else if (im.mode == kModeNan) {
            gap = gap_s = std::numeric_limits<double>::quiet_NaN();
        } else if (im.mode == kModeFdpg) {
            gap_s = std::max(sst.gp, 0.0);
            if (std::isnan(sst.gp)) gap_s = sst.gp;
            gap = im.e ? std::ldexp(gap_s, 2 * im.e) : gap_s;
            it = sst.it;
            if (sst.status != kConverged) notconv = true;
        }
        ws->gaps[(size_t)b] = gap;
        ws->iters[(size_t)b] = it;
        ws->zerrs[(size_t)b] = certified_error(gap_s, im.dd, g.N, im.e, ws->dtype, conj ? 2 : 1);
        gsum += gap;
        imax = std::max(imax, it);
    }
    ws->seeded = false;
    if (inf) return FP_EINVAL;
    ws->dual_valid = true;
    if (keep) ws->valid = true;
    ws->info = fp_info{gsum, imax, 0};
    ws->info_status = notconv ? FP_ENOTCONV : FP_OK;
    ws->info_valid = true;
    if (info) *info = ws->info;
    return ws->info_status;
}

}  // namespace

namespace {

// Elementwise copy between two host arrays of one dtype and shape (any
// strides; dst may be src exactly), or a fill of dst when src is null.
void host_copy(const Arr *src, const Arr &dst, double fill) {
    const int64_t n = dst.numel();
    const size_t T = dst.itemsize();
    std::vector<int64_t> idx((size_t)dst.ndim, 0);
    for (int64_t i = 0; i < n; ++i) {
        int64_t od = 0, os = 0;
        for (int d = 0; d < dst.ndim; ++d) {
            od += idx[(size_t)d] * dst.strides[d];
            if (src) os += idx[(size_t)d] * src->strides[d];
        }
        char *q = dst.data + od * (int64_t)T;
        if (src) std::memmove(q, src->data + os * (int64_t)T, T);
        else if (dst.dtype == FP_F32) *reinterpret_cast<float *>(q) = (float)fill;
        else *reinterpret_cast<double *>(q) = fill;
        for (int d = dst.ndim - 1; d >= 0; --d) {
            if (++idx[(size_t)d] < dst.shape[d]) break;
            idx[(size_t)d] = 0;
        }
    }
}

// dst = src (or the fill) for arrays on the workspace's side: host loops, or
// device copies through `scratch` (dst's size) on the stream.
fp_status copy_or_fill(fp_workspace *ws, const Arr *src, const Arr &dst, double fill, void *scratch) {
    if (dst.numel() == 0) return FP_OK;
    if (ws->host_mode) {
        host_copy(src, dst, fill);
        return FP_OK;
    }
    cudaStream_t s = ws->stream;
    cudaError_t e = cudaSuccess;
    if (src) {
        e = strided_copy(src->data, src->dtype, src->shape, src->strides, dst.ndim, dst.data, dst.dtype, dst.strides, s);
    } else {
        const int64_t n = dst.numel();
        const size_t T = dst.itemsize();
        std::vector<char> h((size_t)n * T);
        for (int64_t i = 0; i < n; ++i) {
            if (T == 4) reinterpret_cast<float *>(h.data())[i] = (float)fill;
            else reinterpret_cast<double *>(h.data())[i] = fill;
        }
        int64_t cst[FP_MAX_NDIM];
        int64_t sz = 1;
        for (int d = dst.ndim - 1; d >= 0; --d) {
            cst[d] = sz;
            sz *= dst.shape[d];
        }
        e = cudaMemcpyAsync(scratch, h.data(), h.size(), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = strided_copy(scratch, dst.dtype, dst.shape, cst, dst.ndim, dst.data, dst.dtype, dst.strides, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e);
}

// A parameter vector of m entries (ndim <= 1) on the host or the device.
fp_status param_array(const fp_array *a, int64_t m, Arr &t) {
    if (fp_status s = to_arr(a, t)) return s;
    if (a->ndim > 1 || t.shape[0] != m) return FP_ESHAPE;
    return FP_OK;
}

// The kept point's geometry and device buffers for the derivatives, and its
// structure, built once per kept call (the reference's TVIso::save,
// src/ops/tv_iso.cpp:551-631, done lazily).
fp_status deriv_prepare(const fp_op *op, fp_workspace *ws, VjpGeom &vg, VjpBuffers &bf) {
    if (op->huber) return FP_EINVAL;  // the derivatives of Huber-smoothed TV are not built
    const Geometry &g0 = ws->g;
    cudaStream_t s = ws->stream;
    const int64_t total = g0.B * g0.N;
    vg = VjpGeom{};
    vg.k = g0.k;
    for (int a = 0; a < 3; ++a) vg.L[a] = g0.L[a];
    vg.S[g0.k - 1] = 1;
    for (int a = g0.k - 2; a >= 0; --a) vg.S[a] = vg.S[a + 1] * vg.L[a + 1];
    for (int a = g0.k; a < 3; ++a) vg.S[a] = 1;
    vg.N = g0.N;
    vg.B = g0.B;
    double wmax_all = 0.0;
    for (int a = 0; a < g0.k; ++a)
        if (g0.L[a] > 1) wmax_all = std::max(wmax_all, op->w[a]);
    double wmax = 0.0;
    int nact = 0;
    vg.act1 = -1;
    for (int a = 0; a < 3; ++a) {
        const bool act = a < g0.k && op->w[a] > 0.0 && g0.L[a] > 1 && op->w[a] >= 1e-100 * wmax_all;
        vg.wa[a] = act ? op->w[a] : 0.0;
        wmax = std::max(wmax, vg.wa[a]);
        if (act) {
            ++nact;
            vg.act1 = a;
        }
    }
    if (nact != 1) vg.act1 = -1;
    vg.wmax = wmax > 0.0 ? wmax : 1.0;
    for (int a = 0; a < 3; ++a) vg.wh[a] = vg.wa[a] / vg.wmax;
    const double eps = ws->dtype == FP_F32 ? (double)std::numeric_limits<float>::epsilon() : 2.2e-16;
    // the flat margin below the radius: the reference's 1e-9, or 64 eps where
    // the iterates are float32 (its device path's dual_eta)
    vg.eta = ws->dtype == FP_F32 ? 64.0 * eps : 1e-9;
    bf = VjpBuffers{};
    bf.d = ws->d;
    bf.U[0] = ws->U[0];
    bf.U[1] = ws->U[1];
    bf.img = ws->img;
    bf.st = ws->st;
    bf.alpha = ws->spatial;
    bf.alpha_stride = 0;
    bf.dtype = ws->dtype;
    bf.flat = ws->v_flat;
    bf.root = ws->v_root;
    bf.cnt = ws->v_cnt;
    bf.gz = ws->v_gz;
    bf.acc = ws->v_acc;
    const size_t bn = (size_t)total;
    bf.b = ws->v_vec;
    bf.x = ws->v_vec + bn;
    bf.r = ws->v_vec + 2 * bn;
    bf.pv = ws->v_vec + 3 * bn;
    bf.qv = ws->v_vec + 4 * bn;
    bf.dinv = ws->v_vec + 5 * bn;
    bf.y = ws->v_vec + 6 * bn;
    bf.h = ws->v_h;
    bf.vimg = ws->v_img;
    bf.cg = ws->v_cg;
    bf.ggam = ws->v_ggam;
    bf.gw = ws->v_gw;
    bf.part = ws->part;
    bf.ticket = ws->ticket;
    bf.live = ws->live;
    bf.err = ws->err;
    bf.max_part = ws->max_part;
    if (!bf.flat) return FP_EINVAL;
    if (op->kind == kAniso) {
        // the anisotropic kept point (tv_aniso.cpp:1012-1180): every axis of
        // extent > 1 carries edges, their weights op->w
        for (int a = 0; a < 3; ++a) {
            vg.w[a] = a < g0.k ? op->w[a] : 0.0;
            vg.bmax[a] = 1.0;
        }
        if (!op->spatial.empty())
            for (int a = 0; a < g0.k; ++a) {
                double m = 0.0;
                for (int64_t i = 0; i < g0.N; ++i) m = std::max(m, op->spatial[(size_t)(a * g0.N + i)]);
                vg.bmax[a] = m;
            }
        vg.eps_t = eps;
        bf.zp = static_cast<const char *>(ws->U[1]) + (size_t)total * (ws->dtype == FP_F32 ? 4 : 8);
        bf.qd = ws->dual;
        bf.beta = ws->spatial;
        bf.aimg = ws->an_img;
        bf.ast = ws->an_st;
        bf.avimg = reinterpret_cast<AnVjpImage *>(ws->v_img);
        bf.code = ws->v_code;
        bf.side = ws->branch_on ? ws->v_side : nullptr;
        vg.stol = ws->branch_tol;
        if (ws->struct_valid) return FP_OK;
        auto *hv = reinterpret_cast<AnVjpImage *>(ws->h_vimg);
        for (int64_t b = 0; b < g0.B; ++b) {
            const AnImage &im = ws->h_an_img[b];
            const AnState &st = ws->h_an_st[b];
            AnVjpImage &vi = hv[b];
            vi.gamma = im.gamma_in;
            vi.gap = (im.mode == kAnAdbpg || im.mode == kAnFdpg3) ? std::max(st.gp, 0.0) : 0.0;
            vi.tau = vi.tau0 = 0.0;
        }
        cudaError_t e = cudaMemcpyAsync(ws->v_img, hv, (size_t)g0.B * sizeof(AnVjpImage), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = an_vjp_structure(ws->dtype, vg, bf, s);
        if (e != cudaSuccess) return cuda_status(e);
        ws->struct_valid = true;
        return FP_OK;
    }
    if (ws->struct_valid) return FP_OK;
    // per image, from the forward (tv_iso.cpp:559-570), at the solved scale
    for (int64_t b = 0; b < g0.B; ++b) {
        const IsoImage &im = ws->h_img[b];
        const IsoState &st = ws->h_st[b];
        VjpImage &vi = ws->h_vimg[b];
        const bool from_dual = im.mode == kModeFdpg;
        const double gap_s = im.mode == kModeFdpg ? std::max(st.gp, 0.0) : 0.0;
        vi.gs = std::ldexp(im.gamma_in, -im.e);
        vi.rel = im.dd > 0.0 ? std::sqrt(2.0 * gap_s / im.dd) : 0.0;
        vi.mu = from_dual ? 0.1 * vg.wmax * std::sqrt(2.0 * gap_s / (double)g0.N) : 0.0;
        vi.thr = from_dual ? vg.wmax * 64.0 * eps * std::ldexp(im.maxabs, -im.e) : 0.0;
    }
    cudaError_t e = cudaMemcpyAsync(ws->v_img, ws->h_vimg, (size_t)g0.B * sizeof(VjpImage), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = vjp_structure(ws->dtype, vg, bf, s);
    if (e != cudaSuccess) return cuda_status(e);
    ws->struct_valid = true;
    return FP_OK;
}

// An input image batch (cotangent or tangent) as a contiguous device array:
// itself, or a copy in `stage`.
fp_status stage_input(fp_workspace *ws, const Arr &a, void *stage, const void **dev) {
    cudaStream_t s = ws->stream;
    const int64_t total = a.numel();
    const size_t T = a.itemsize();
    cudaError_t e = cudaSuccess;
    if (ws->host_mode) {
        std::vector<char> tmp((size_t)total * T);
        Arr c = a;
        int64_t cst[FP_MAX_NDIM];
        int64_t sz = 1;
        for (int d = a.ndim - 1; d >= 0; --d) {
            cst[d] = sz;
            sz *= a.shape[d];
        }
        c.data = tmp.data();
        for (int d = 0; d < a.ndim; ++d) c.strides[d] = cst[d];
        host_copy(&a, c, 0.0);
        e = cudaMemcpyAsync(stage, tmp.data(), tmp.size(), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        *dev = stage;
    } else if (a.contiguous()) {
        if (pointer_device(a.data) != ws->device) return FP_EINVAL;
        *dev = a.data;
    } else {
        if (pointer_device(a.data) != ws->device) return FP_EINVAL;
        int64_t cst[FP_MAX_NDIM];
        int64_t sz = 1;
        for (int d = a.ndim - 1; d >= 0; --d) {
            cst[d] = sz;
            sz *= a.shape[d];
        }
        e = strided_copy(a.data, a.dtype, a.shape, a.strides, a.ndim, stage, a.dtype, cst, s);
        *dev = stage;
    }
    return cuda_status(e);
}

// The result image batch from the contiguous device buffer `res` into out
// (nothing to do when res is out itself).
fp_status unstage_output(fp_workspace *ws, const void *res, const Arr &out) {
    if (res == out.data) return FP_OK;
    cudaStream_t s = ws->stream;
    const int64_t total = out.numel();
    const size_t T = out.itemsize();
    int64_t cst[FP_MAX_NDIM];
    int64_t sz = 1;
    for (int d = out.ndim - 1; d >= 0; --d) {
        cst[d] = sz;
        sz *= out.shape[d];
    }
    cudaError_t e;
    if (ws->host_mode) {
        std::vector<char> tmp((size_t)total * T);
        e = cudaMemcpyAsync(tmp.data(), res, tmp.size(), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e);
        Arr c = out;
        c.data = tmp.data();
        for (int d = 0; d < out.ndim; ++d) c.strides[d] = cst[d];
        host_copy(&c, out, 0.0);
        return FP_OK;
    }
    e = strided_copy(res, out.dtype, out.shape, cst, out.ndim, out.data, out.dtype, out.strides, s);
    return cuda_status(e);
}

// The derivative's residual and iterations over the images.
fp_status read_cg(fp_workspace *ws, int64_t nl) {
    cudaStream_t s = ws->stream;
    const int64_t B = ws->g.B;
    cudaError_t e = cudaMemcpyAsync(ws->h_cg, ws->v_cg, (size_t)B * sizeof(CgState), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    double res = 0.0;
    int its = 0;
    for (int64_t b = 0; b < B; ++b) {
        res = std::max(res, ws->h_cg[b].res);
        its = std::max(its, ws->h_cg[b].it);
    }
    ws->deriv_residual = res;
    ws->deriv_iters = its;
    ws->kernel_launches = nl;
    return FP_OK;
}

// The derivative at the kept point (the reference's vjp_impl,
// src/api/api.cpp:693-738, and image_vjp_driver, src/core/driver.hpp:1505-1560):
// gx = J^T g, the step's gradient and the parameters' (axis weights, then
// pixel weights), each summed over the batch. Isotropic TV.
fp_status vjp_impl(const fp_op *op, fp_workspace *ws, const fp_array *ga, fp_array *gxa, double *ggamma,
                   fp_array *ggdev, fp_array *gpa) {
    if (!op || !ws || !ga || !gxa) return FP_EINVAL;
    if (ws->op != op || !ws->valid) return FP_EINVAL;
    Arr g, gx;
    if (fp_status s = to_arr(ga, g)) return s;
    if (fp_status s = to_arr(gxa, gx)) return s;
    if (g.dtype != ws->dtype || gx.dtype != ws->dtype) return FP_EDTYPE;
    if (g.ndim != ws->ndim || gx.ndim != ws->ndim) return FP_ESHAPE;
    for (int d = 0; d < ws->ndim; ++d)
        if (g.shape[d] != ws->shape[d] || gx.shape[d] != ws->shape[d]) return FP_ESHAPE;
    if (fp_status s = check_output(&g, gx)) return s;
    if (g.device != gx.device || ws->host_mode != (g.device == FP_DEVICE_CPU)) return FP_EINVAL;
    const int64_t P = fp_op_nparams(op);
    Arr gp;
    if (gpa)  // validated before any work
        if (fp_status s = param_array(gpa, P, gp)) return s;
    Arr gg;
    if (ggdev) {
        if (fp_status s = to_arr(ggdev, gg)) return s;
        if (gg.device != FP_DEVICE_CUDA || gg.numel() != 1) return FP_EINVAL;
    }
    const Geometry &g0 = ws->g;
    DeviceScope dsc(ws->device);
    cudaStream_t s = ws->stream;
    std::vector<double> tot((size_t)P, 0.0);
    double gsum = 0.0;
    auto finish = [&]() -> fp_status {
        // the step's and the parameters' gradients to the caller
        if (ggamma) *ggamma = gsum;
        cudaError_t e = cudaSuccess;
        if (ggdev) {
            if (gg.dtype == FP_F32) {
                const float v = (float)gsum;
                e = cudaMemcpyAsync(gg.data, &v, sizeof v, cudaMemcpyHostToDevice, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            } else {
                e = cudaMemcpyAsync(gg.data, &gsum, sizeof gsum, cudaMemcpyHostToDevice, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            }
            if (e != cudaSuccess) return cuda_status(e);
        }
        if (!gpa || P == 0) return FP_OK;
        if (gp.device == FP_DEVICE_CPU) {
            for (int64_t i = 0; i < P; ++i) {
                char *q = gp.data + i * gp.strides[0] * (int64_t)gp.itemsize();
                if (gp.dtype == FP_F32) *reinterpret_cast<float *>(q) = (float)tot[(size_t)i];
                else *reinterpret_cast<double *>(q) = tot[(size_t)i];
            }
            return FP_OK;
        }
        if (pointer_device(gp.data) != ws->device) return FP_EINVAL;
        // through the derivative scratch (7 B N >= k + N doubles)
        double *scr = ws->v_vec;
        if (!scr) return FP_EINVAL;
        const int64_t one = 1, shp = P;
        e = cudaMemcpyAsync(scr, tot.data(), (size_t)P * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = strided_copy(scr, FP_F64, &shp, &one, 1, gp.data, gp.dtype, gp.strides, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        return cuda_status(e);
    };
    ws->vjp_gg_img.assign((size_t)g0.B, 0.0);
    ws->vjp_gw_img.assign((size_t)(g0.B * op->k), 0.0);
    if (ws->identity) {  // gx = g; no parameter gradient; the sigma-derivative NaN (api.cpp:711-716)
        if (fp_status st = copy_or_fill(ws, &g, gx, 0.0, nullptr)) return st;
        gsum = std::numeric_limits<double>::quiet_NaN();
        ws->vjp_gg_img.assign((size_t)g0.B, gsum);
        return finish();
    }
    if (g0.B * g0.N == 0) return finish();
    VjpGeom vg;
    VjpBuffers bf;
    if (fp_status st = deriv_prepare(op, ws, vg, bf)) return st;
    // the cotangent and the output, contiguous on the device (the V buffers
    // are free after the solve)
    const void *gsrc = nullptr;
    if (fp_status st = stage_input(ws, g, ws->V[0], &gsrc)) return st;
    const bool direct = !ws->host_mode && gx.contiguous();
    void *gdst = direct ? gx.data : ws->V[1];
    if (direct && pointer_device(gx.data) != ws->device) return FP_EINVAL;
    const bool params = gpa && P > 0;
    int64_t nl = 0;
    if (op->kind == kAniso) {
        // component averages, no linear solve (tv_aniso.cpp:1398-1440)
        const int64_t nb = P - op->k;  // edge weights
        std::vector<double> gb((size_t)std::max<int64_t>(nb, 0));
        cudaError_t e = an_vjp_solve(ws->dtype, vg, bf, gsrc, gdst, ws->conj ? 1 : 0, true,
                                     (params && nb > 0) ? gb.data() : nullptr, s, &nl);
        if (e != cudaSuccess) return cuda_status(e);
        if (fp_status st = unstage_output(ws, gdst, gx)) return st;
        e = cudaMemcpyAsync(ws->h_gw, ws->v_gw, (size_t)g0.B * 3 * sizeof(double), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e);
        // d/dw_a = -gamma sum_C S_{C,a} g_C; d/dgamma = -sum_a w_a sum_C S_{C,a} g_C
        const auto *hv = reinterpret_cast<const AnVjpImage *>(ws->h_vimg);
        ws->vjp_gg_img.assign((size_t)g0.B, 0.0);
        ws->vjp_gw_img.assign((size_t)(g0.B * op->k), 0.0);
        for (int64_t b = 0; b < g0.B; ++b)
            for (int a = 0; a < op->k; ++a) {
                tot[(size_t)a] -= hv[b].gamma * ws->h_gw[3 * b + a];
                gsum -= op->w[a] * ws->h_gw[3 * b + a];
                ws->vjp_gg_img[(size_t)b] -= ws->conj ? 0.0 : op->w[a] * ws->h_gw[3 * b + a];
                ws->vjp_gw_img[(size_t)(b * op->k + a)] = (ws->conj ? 1.0 : -1.0) * hv[b].gamma * ws->h_gw[3 * b + a];
            }
        if (params) {
            for (int64_t i = 0; i < nb; ++i) tot[(size_t)(op->k + i)] = gb[(size_t)i];
            if (ws->conj)
                for (double &v : tot) v = -v;
        }
        if (ws->conj) gsum = 0.0;  // y - prox(y) is constant in sigma
        ws->deriv_residual = 0.0;
        ws->deriv_iters = 0;
        ws->kernel_launches = nl;
        return finish();
    }
    cudaError_t e = vjp_solve(ws->dtype, vg, bf, gsrc, gdst, ws->deriv_tol, ws->deriv_max_iter, ws->conj ? 1 : 0,
                              params, s, ws->h_live, ws->ev[0], &nl);
    if (e != cudaSuccess) return cuda_status(e);
    if (fp_status st = unstage_output(ws, gdst, gx)) return st;
    e = cudaMemcpyAsync(ws->h_ggam, ws->v_ggam, (size_t)g0.B * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && params)
        e = cudaMemcpyAsync(ws->h_gw, ws->v_gw, (size_t)g0.B * 3 * sizeof(double), cudaMemcpyDeviceToHost, s);
    std::vector<double> ga_host;
    const int64_t na = P - op->k;  // pixel weights
    if (e == cudaSuccess && params && na > 0) {
        ga_host.resize((size_t)na);
        e = cudaMemcpyAsync(ga_host.data(), bf.qv, (size_t)na * sizeof(double), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    ws->vjp_gg_img.assign((size_t)g0.B, 0.0);
    ws->vjp_gw_img.assign((size_t)(g0.B * op->k), 0.0);
    for (int64_t b = 0; b < g0.B; ++b) {
        gsum += ws->h_ggam[b];
        ws->vjp_gg_img[(size_t)b] = ws->h_ggam[b];
    }
    if (params) {
        for (int a = 0; a < op->k; ++a)
            for (int64_t b = 0; b < g0.B; ++b) {
                tot[(size_t)a] += ws->h_gw[3 * b + a];
                ws->vjp_gw_img[(size_t)(b * op->k + a)] = (ws->conj ? -1.0 : 1.0) * ws->h_gw[3 * b + a];
            }
        for (int64_t i = 0; i < na; ++i) tot[(size_t)(op->k + i)] = ga_host[(size_t)i];
        // the conjugate y - prox(y): -sigma times the parameters' gradients,
        // sigma = 1 for TV (api.cpp:726-730)
        if (ws->conj)
            for (double &v : tot) v = -v;
    }
    if (fp_status st = read_cg(ws, nl)) return st;
    return finish();
}

// dout = J_x dx + (dz/dgamma) dgamma + (dz/dtheta) dtheta at the kept point
// (the reference's jvp_impl, src/api/api.cpp:583-616, image_jvp_driver,
// src/core/driver.hpp:1448-1503, and TVIso::jvp_img, src/ops/tv_iso.cpp:953-997).
// Isotropic TV.
fp_status jvp_impl(const fp_op *op, fp_workspace *ws, const fp_array *dxa, double dgamma, const fp_array *dpa,
                   fp_array *oa) {
    if (!op || !ws || !oa) return FP_EINVAL;
    if (ws->op != op || !ws->valid) return FP_EINVAL;
    if (!std::isfinite(dgamma)) return FP_EPARAM;
    Arr dx, out;
    if (fp_status s = to_arr(oa, out)) return s;
    auto like_ws = [&](const Arr &a) {
        if (a.dtype != ws->dtype) return FP_EDTYPE;
        if (a.ndim != ws->ndim) return FP_ESHAPE;
        for (int d = 0; d < a.ndim; ++d)
            if (a.shape[d] != ws->shape[d]) return FP_ESHAPE;
        return FP_OK;
    };
    if (fp_status s = like_ws(out)) return s;
    if (dxa) {
        if (fp_status s = to_arr(dxa, dx)) return s;
        if (fp_status s = like_ws(dx)) return s;
    }
    if (fp_status s = check_output(dxa ? &dx : nullptr, out)) return s;
    const int64_t P = fp_op_nparams(op);
    Arr dp;
    const bool has_dp = dpa && P > 0;
    if (has_dp)
        if (fp_status s = param_array(dpa, P, dp)) return s;
    if (ws->host_mode != (out.device == FP_DEVICE_CPU)) return FP_EINVAL;
    if (dxa && dx.device != out.device) return FP_EINVAL;
    DeviceScope dsc(ws->device);
    if (ws->identity)  // J = I; the sigma-derivative NaN (api.cpp:603-607)
        return copy_or_fill(ws, dgamma != 0.0 ? nullptr : (dxa ? &dx : nullptr), out,
                            dgamma != 0.0 ? std::numeric_limits<double>::quiet_NaN() : 0.0, ws->V[1]);
    const Geometry &g0 = ws->g;
    if (g0.B * g0.N == 0) return FP_OK;
    if (ws->conj) dgamma = 0.0;  // y - prox(y) is constant in sigma for TV (api.cpp:610)
    cudaStream_t s = ws->stream;
    VjpGeom vg;
    VjpBuffers bf;
    if (fp_status st = deriv_prepare(op, ws, vg, bf)) return st;
    // the parameter direction: the axis weights on the host, the pixel (or
    // edge) weights as doubles on the device, in qv (N) for isotropic TV and
    // h (k N) for anisotropic TV (both free until the solve)
    JvpDir dir{{0.0, 0.0, 0.0}};
    const double *dalpha = nullptr;
    const int64_t na = P - op->k;
    double *dtail = op->kind == kAniso ? bf.h : bf.qv;
    cudaError_t e = cudaSuccess;
    if (has_dp) {
        if (dp.device == FP_DEVICE_CPU) {
            std::vector<double> v((size_t)P);
            for (int64_t i = 0; i < P; ++i) {
                const char *q = dp.data + i * dp.strides[0] * (int64_t)dp.itemsize();
                v[(size_t)i] = dp.dtype == FP_F32 ? (double)*reinterpret_cast<const float *>(q)
                                                  : *reinterpret_cast<const double *>(q);
            }
            for (int a = 0; a < op->k; ++a) dir.dw[a] = v[(size_t)a];
            if (na > 0) e = cudaMemcpyAsync(dtail, v.data() + op->k, (size_t)na * sizeof(double),
                                            cudaMemcpyHostToDevice, s);
        } else {
            if (pointer_device(dp.data) != ws->device) return FP_EINVAL;
            const int64_t one = 1, kk = op->k;
            double hw[3] = {0.0, 0.0, 0.0};
            e = strided_copy(dp.data, dp.dtype, &kk, dp.strides, 1, bf.b, FP_F64, &one, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(hw, bf.b, (size_t)kk * sizeof(double), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess && na > 0)
                e = strided_copy(dp.data + kk * dp.strides[0] * (int64_t)dp.itemsize(), dp.dtype, &na, dp.strides, 1,
                                 dtail, FP_F64, &one, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            for (int a = 0; a < op->k; ++a) dir.dw[a] = hw[a];
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e);
        for (int a = 0; a < op->k; ++a)
            if (!std::isfinite(dir.dw[a])) return FP_EPARAM;
        if (na > 0) dalpha = dtail;
    }
    const void *dsrc = nullptr;
    if (dxa)
        if (fp_status st = stage_input(ws, dx, ws->V[0], &dsrc)) return st;
    const bool direct = !ws->host_mode && out.contiguous();
    void *ddst = direct ? out.data : ws->V[1];
    if (direct && pointer_device(out.data) != ws->device) return FP_EINVAL;
    int64_t nl = 0;
    if (op->kind == kAniso) {
        e = an_jvp_solve(ws->dtype, vg, bf, dsrc, ddst, dgamma, dir, dalpha, ws->conj ? 1 : 0, s, &nl);
        if (e != cudaSuccess) return cuda_status(e);
        if (fp_status st = unstage_output(ws, ddst, out)) return st;
        e = cudaStreamSynchronize(s);
        ws->deriv_residual = 0.0;
        ws->deriv_iters = 0;
        ws->kernel_launches = nl;
        return cuda_status(e);
    }
    e = jvp_solve(ws->dtype, vg, bf, dsrc, ddst, dgamma, dir, dalpha, ws->deriv_tol, ws->deriv_max_iter,
                  ws->conj ? 1 : 0, s, ws->h_live, ws->ev[0], &nl);
    if (e != cudaSuccess) return cuda_status(e);
    if (fp_status st = unstage_output(ws, ddst, out)) return st;
    return read_cg(ws, nl);
}

// fp_workspace_refine (the reference's refine_impl, api.cpp:1182-1216): the
// kept call solved again from its saved input (d at the input's scale) and,
// warm, from its dual, to tol; the derivatives, the dual and the call's
// results then describe the refined point. The input is rebuilt in V[1] and
// a result nobody asked for goes to V[0]: neither is read by the solve after
// its set-up, nor by the derivatives after it.
fp_status refine_impl(const fp_op *op, fp_workspace *ws, double tol, int max_iter, fp_array *oa, fp_info *info) {
    if (!op || !ws || ws->op != op || !ws->valid || !ws->keep) return FP_EINVAL;
    if (!(tol >= 0.0) || !std::isfinite(tol) || max_iter < 1) return FP_EPARAM;
    Arr out;
    if (oa) {
        if (fp_status s = to_arr(oa, out)) return s;
        if (out.dtype != ws->dtype) return FP_EDTYPE;
        if (out.ndim != ws->ndim) return FP_ESHAPE;
        for (int d = 0; d < out.ndim; ++d)
            if (out.shape[d] != ws->shape[d]) return FP_ESHAPE;
        if (fp_status s = check_output(nullptr, out)) return s;
    }
    if (ws->identity) return oa ? FP_EINVAL : FP_OK;  // sigma = 0 saved no input to refine
    const Geometry &g0 = ws->g;
    const int64_t total = g0.B * g0.N;
    if (total == 0) return FP_OK;
    DeviceScope dsc(ws->device);
    cudaStream_t s = ws->stream;
    const bool aniso = op->kind == kAniso;
    const bool conj = ws->conj;
    // the saved input: d 2^e per image, into V[1]
    std::vector<int> ex((size_t)g0.B);
    std::vector<double> steps((size_t)g0.B);
    for (int64_t b = 0; b < g0.B; ++b) {
        ex[(size_t)b] = aniso ? ws->h_an_img[b].e : ws->h_img[b].e;
        steps[(size_t)b] = aniso ? ws->h_an_img[b].gamma_in : ws->h_img[b].gamma_in;
    }
    cudaError_t e = cudaMemcpyAsync(ws->lmap, ex.data(), ex.size() * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = unscale_images(ws->dtype, ws->d, ws->lmap, g0.N, g0.B, ws->V[1], s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    const size_t T = ws->dtype == FP_F32 ? 4 : 8;
    std::vector<char> hx, hz;
    fp_array xa{}, za{}, sa{};
    xa.dtype = (fp_dtype)ws->dtype;
    xa.ndim = ws->ndim;
    xa.shape = ws->shape;
    xa.strides = nullptr;
    za = xa;
    if (ws->host_mode) {
        hx.resize((size_t)total * T);
        e = cudaMemcpyAsync(hx.data(), ws->V[1], hx.size(), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e);
        xa.data = hx.data();
        xa.device = FP_DEVICE_CPU;
        if (!oa) hz.resize(hx.size());
        za.data = hz.data();
        za.device = FP_DEVICE_CPU;
    } else {
        xa.data = ws->V[1];
        xa.device = FP_DEVICE_CUDA;
        za.data = ws->V[0];
        za.device = FP_DEVICE_CUDA;
    }
    fp_options o{};
    fp_options_init(&o);
    o.tol = tol;
    o.max_iter = max_iter;
    o.keep_structure = 1;
    const int64_t one = (int64_t)g0.B;
    const int64_t bshape[1] = {one};
    sa.data = steps.data();
    sa.dtype = FP_F64;
    sa.ndim = 1;
    sa.shape = bshape;
    sa.strides = nullptr;
    sa.device = FP_DEVICE_CPU;
    // the steps per image over the batch shape
    std::vector<int64_t> bsh((size_t)std::max(1, ws->ndim - g0.k));
    const bool batched = ws->ndim > g0.k;
    if (batched) {
        for (int d = 0; d < ws->ndim - g0.k; ++d) bsh[(size_t)d] = ws->shape[d];
        sa.ndim = ws->ndim - g0.k;
        sa.shape = bsh.data();
    }
    const bool was_warm = ws->warm;
    ws->warm = true;
    fp_info local{0.0, 0, 0};
    fp_status st;
    fp_array *outp = oa ? oa : &za;
    if (conj) st = prox_impl(op, 1.0, &xa, outp, &o, ws, info ? info : &local, true, nullptr);
    else if (batched) st = prox_impl(op, 0.0, &xa, outp, &o, ws, info ? info : &local, false, &sa);
    else st = prox_impl(op, steps[0], &xa, outp, &o, ws, info ? info : &local, false, nullptr);
    ws->warm = was_warm;
    return st;
}

// ---- structure of the derivative (the reference's api.cpp:1032-1180; its
// queries refuse device workspaces, which this library answers) ----

fp_status struct_ws(const fp_workspace *ws) {
    if (!ws || !ws->op || !ws->keep || !ws->valid) return FP_EINVAL;
    return FP_OK;
}

int64_t struct_units(const fp_workspace &ws) { return ws.g.B * ws.g.N == 0 ? 0 : ws.g.B; }

// An output array of the queries: x's shape, of its dtype class (Float: x's dtype).
fp_status struct_out(const fp_workspace &ws, const fp_array *a, Arr &out, Dt kind) {
    if (fp_status s = to_arr(a, out, kind)) return s;
    if (kind == Dt::Float && out.dtype != ws.dtype) return FP_EDTYPE;
    if (out.ndim != ws.ndim) return FP_ESHAPE;
    for (int d = 0; d < out.ndim; ++d)
        if (out.shape[d] != ws.shape[d]) return FP_ESHAPE;
    if (out.numel() > 0 && out.device == FP_DEVICE_CUDA && pointer_device(out.data) != ws.device) return FP_EINVAL;
    return FP_OK;
}

// Writes host values (C order, out's element size) into out, on the host or
// the device (through the workspace's V[0] and a scatter).
fp_status put_array(fp_workspace *ws, const Arr &out, const std::vector<char> &h) {
    const int64_t n = out.numel();
    if (n == 0) return FP_OK;
    const size_t es = out.itemsize();
    if (out.device == FP_DEVICE_CPU) {
        std::vector<int64_t> idx((size_t)out.ndim, 0);
        for (int64_t i = 0; i < n; ++i) {
            int64_t o = 0;
            for (int d = 0; d < out.ndim; ++d) o += idx[(size_t)d] * out.strides[d];
            std::memcpy(out.data + o * (int64_t)es, h.data() + i * (int64_t)es, es);
            for (int d = out.ndim - 1; d >= 0; --d) {
                if (++idx[(size_t)d] < out.shape[d]) break;
                idx[(size_t)d] = 0;
            }
        }
        return FP_OK;
    }
    cudaStream_t s = ws->stream;
    cudaError_t e;
    if (out.contiguous()) {
        e = cudaMemcpyAsync(out.data, h.data(), h.size(), cudaMemcpyHostToDevice, s);
    } else {
        e = cudaMemcpyAsync(ws->V[0], h.data(), h.size(), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = scatter_elements(ws->V[0], es, out.ndim, out.shape, out.strides, out.data, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return cuda_status(e);
}

template <class V>
std::vector<char> filled(int64_t n, V v) {
    std::vector<char> h((size_t)n * sizeof(V));
    for (int64_t i = 0; i < n; ++i) std::memcpy(h.data() + i * (int64_t)sizeof(V), &v, sizeof(V));
    return h;
}

// The kept point's structure on the device, and its geometry (for an
// isotropic point also the weights and the dual, which the kink test reads).
fp_status struct_prepare(fp_workspace *ws, VjpGeom &vg, VjpBuffers &bf) {
    const fp_op *op = ws->op;
    if (fp_status st = deriv_prepare(op, ws, vg, bf)) return st;
    for (int a = 0; a < 3; ++a) vg.w[a] = a < ws->g.k ? op->w[a] : 0.0;
    bf.qd = ws->dual;
    return FP_OK;
}

fp_status units_impl(const fp_workspace *ws, int64_t *count, int64_t *size) {
    if (fp_status s = struct_ws(ws)) return s;
    if (count) *count = struct_units(*ws);
    if (size) *size = ws->g.N;
    return FP_OK;
}

fp_status states_impl(fp_workspace *ws, fp_array *sa, int64_t *nfixed) {
    if (fp_status s = struct_ws(ws)) return s;
    Arr st;
    if (sa)
        if (fp_status s = struct_out(*ws, sa, st, Dt::Int8)) return s;
    // every entry of a TV solution moves with its region; after the
    // conjugate at sigma = 0 the inner prox's Jacobian I - J is 0
    const int64_t total = ws->g.B * ws->g.N;
    const int8_t v = ws->identity ? (int8_t)FP_ENTRY_ZERO : (int8_t)FP_ENTRY_FREE;
    if (sa)
        if (fp_status s = put_array(ws, st, filled<int8_t>(total, v))) return s;
    if (nfixed) *nfixed = ws->identity ? total : 0;
    return FP_OK;
}

fp_status regions_impl(fp_workspace *ws, fp_array *la, fp_array *ga, int64_t *nregions, int64_t count) {
    if (fp_status s = struct_ws(ws)) return s;
    const int64_t units = struct_units(*ws);
    if (nregions && count != units) return FP_ESHAPE;
    Arr lab, sg;
    if (la) {
        if (fp_status s = struct_out(*ws, la, lab, Dt::Label)) return s;
        if (lab.dtype == FP_I32 && ws->g.N > std::numeric_limits<int32_t>::max()) return FP_ESHAPE;
    }
    if (ga)
        if (fp_status s = struct_out(*ws, ga, sg, Dt::Int8)) return s;
    const Geometry &g0 = ws->g;
    const int64_t total = g0.B * g0.N;
    if (total == 0) return FP_OK;
    DeviceScope dsc(ws->device);
    std::vector<int32_t> hl((size_t)total, -1);
    std::vector<double> hn((size_t)g0.B, 0.0);
    if (!ws->identity) {
        VjpGeom vg;
        VjpBuffers bf;
        if (fp_status st = struct_prepare(ws, vg, bf)) return st;
        cudaStream_t s = ws->stream;
        int32_t *dl = static_cast<int32_t *>(ws->V[1]);
        double *dn = ws->v_ggam;
        cudaError_t e = query_labels(ws->op->kind == kAniso, vg, bf, dl, dn, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hl.data(), dl, (size_t)total * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hn.data(), dn, (size_t)g0.B * 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e);
    }
    if (nregions)
        for (int64_t b = 0; b < g0.B; ++b) nregions[b] = (int64_t)hn[(size_t)b];
    if (la) {
        std::vector<char> h((size_t)total * lab.itemsize());
        for (int64_t i = 0; i < total; ++i) {
            if (lab.dtype == FP_I32) std::memcpy(h.data() + i * 4, &hl[(size_t)i], 4);
            else {
                const int64_t v = hl[(size_t)i];
                std::memcpy(h.data() + i * 8, &v, 8);
            }
        }
        if (fp_status st = put_array(ws, lab, h)) return st;
    }
    if (ga) {
        std::vector<char> h((size_t)total);
        for (int64_t i = 0; i < total; ++i) h[(size_t)i] = (char)(hl[(size_t)i] >= 0 ? 1 : 0);
        if (fp_status st = put_array(ws, sg, h)) return st;
    }
    return FP_OK;
}

fp_status constraint_impl(fp_workspace *ws, fp_array *ca, int8_t *active, int64_t count) {
    if (fp_status s = struct_ws(ws)) return s;
    if (active && count != struct_units(*ws)) return FP_ESHAPE;
    Arr c;
    if (ca)
        if (fp_status s = struct_out(*ws, ca, c, Dt::Float)) return s;
    // TV has no linear constraint
    if (active) std::fill(active, active + count, int8_t{0});
    if (ca) {
        const int64_t total = ws->g.B * ws->g.N;
        if (ws->dtype == FP_F32) return put_array(ws, c, filled<float>(total, 0.0f));
        return put_array(ws, c, filled<double>(total, 0.0));
    }
    return FP_OK;
}

// Every image's derivative exact, and the largest curvature cap of the
// isotropic derivative in the units of x (the reference's api.cpp:1219-1232).
fp_status deriv_exact_impl(const fp_workspace *ws, int *exact, double *smoothing) {
    if (!ws || !ws->valid || !ws->keep) return FP_EINVAL;
    int all = 1;
    double mu = 0.0;
    const Geometry &g0 = ws->g;
    if (!ws->identity && g0.B * g0.N != 0) {
        if (ws->op->kind == kAniso) {
            for (int64_t b = 0; b < g0.B; ++b) {
                const AnImage &im = ws->h_an_img[b];
                if ((im.mode == kAnAdbpg || im.mode == kAnFdpg3) && !ws->h_an_st[b].polished) all = 0;
            }
        } else {
            // mu = 0.1 wmax sqrt(2 gap / N) at the solved scale (tv_iso.cpp:566-568)
            double wmax = 0.0;
            for (int a = 0; a < g0.k; ++a)
                if (ws->op->w[a] > 0.0 && g0.L[a] > 1) wmax = std::max(wmax, ws->op->w[a]);
            for (int64_t b = 0; b < g0.B; ++b) {
                const IsoImage &im = ws->h_img[b];
                if (im.mode != kModeFdpg) continue;
                const double m = 0.1 * wmax * std::sqrt(2.0 * std::max(ws->h_st[b].gp, 0.0) / (double)g0.N);
                if (m > 0.0) all = 0;
                mu = std::max(mu, std::ldexp(m, im.e));
            }
        }
    }
    if (exact) *exact = all;
    if (smoothing) *smoothing = mu;
    return FP_OK;
}

// The kept point's kink mask (FP_I8, x's shape) and the number of entries at
// a kink (the reference's kinks_impl, api.cpp:857-875).
fp_status kinks_impl(fp_workspace *ws, double tol, fp_array *ma, int64_t *count) {
    if (!(tol >= 0.0) || !std::isfinite(tol)) return FP_EPARAM;
    if (!ws || !ws->op || !ws->keep || !ws->valid) return FP_EINVAL;
    Arr m;
    if (ma)
        if (fp_status s = struct_out(*ws, ma, m, Dt::Int8)) return s;
    const Geometry &g0 = ws->g;
    const int64_t total = g0.B * g0.N;
    std::vector<char> h((size_t)total, 0);
    int64_t c = 0;
    if (!ws->identity && total != 0) {
        DeviceScope dsc(ws->device);
        VjpGeom vg;
        VjpBuffers bf;
        if (fp_status st = struct_prepare(ws, vg, bf)) return st;
        const bool aniso = ws->op->kind == kAniso;
        std::vector<double> gam((size_t)g0.B);
        for (int64_t b = 0; b < g0.B; ++b) gam[(size_t)b] = aniso ? ws->h_an_img[b].gamma_in : ws->h_img[b].gamma_in;
        cudaStream_t s = ws->stream;
        // the steps into the structure's scratch (b, free between derivative calls)
        cudaError_t e = cudaMemcpyAsync(bf.b, gam.data(), gam.size() * 8, cudaMemcpyHostToDevice, s);
        int8_t *dm = static_cast<int8_t *>(ws->V[1]);
        if (e == cudaSuccess) e = query_kinks(ws->dtype, aniso, vg, bf, bf.b, tol, dm, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), dm, (size_t)total, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_status(e);
        for (int64_t i = 0; i < total; ++i) c += h[(size_t)i] != 0;
    }
    if (ma)
        if (fp_status st = put_array(ws, m, h)) return st;
    if (count) *count = c;
    return FP_OK;
}

// A branch override for the derivatives of an anisotropic kept point (the
// reference's set_branch_impl, api.cpp:993-1028): the structure is rebuilt
// with side applied at the kinks found with tol; NULL clears it.
fp_status set_branch_impl(fp_workspace *ws, const fp_array *sa, double tol) {
    if (!sa) {
        if (!ws || !ws->op) return FP_EINVAL;
        if (ws->branch_on) ws->struct_valid = false;
        ws->branch_on = false;
        return FP_OK;
    }
    if (!(tol >= 0.0) || !std::isfinite(tol)) return FP_EPARAM;
    if (!ws || !ws->op || !ws->keep) return FP_EINVAL;
    if (ws->op->kind != kAniso) return FP_EINVAL;  // isotropic TV has no branches
    if (!ws->valid) return FP_EINVAL;
    Arr a;
    if (fp_status s = to_arr(sa, a, Dt::Int8)) return s;
    if (a.ndim != ws->ndim) return FP_ESHAPE;
    for (int d = 0; d < a.ndim; ++d)
        if (a.shape[d] != ws->shape[d]) return FP_ESHAPE;
    const int64_t total = ws->g.B * ws->g.N;
    if (ws->identity || total == 0) return FP_OK;
    // the sides in C order, checked before the workspace changes
    std::vector<int8_t> h((size_t)total);
    DeviceScope dsc(ws->device);
    cudaStream_t s = ws->stream;
    {
        std::vector<int64_t> idx((size_t)a.ndim, 0);
        const bool dev = a.device == FP_DEVICE_CUDA;
        std::vector<int8_t> whole;
        int64_t lo = 0, span = 1;
        if (dev) {
            // the array's byte range to the host, then read by its strides
            for (int d = 0; d < a.ndim; ++d) {
                if (a.shape[d] < 2) continue;
                const int64_t e = (a.shape[d] - 1) * a.strides[d];
                if (e < 0) lo += e;
                else span += e;
            }
            span -= lo;
            whole.resize((size_t)span);
            cudaError_t e = cudaMemcpyAsync(whole.data(), a.data + lo, (size_t)span, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) return cuda_status(e);
        }
        for (int64_t i = 0; i < total; ++i) {
            int64_t o = 0;
            for (int d = 0; d < a.ndim; ++d) o += idx[(size_t)d] * a.strides[d];
            const int8_t v = dev ? whole[(size_t)(o - lo)] : reinterpret_cast<const int8_t *>(a.data)[o];
            if (v < -1 || v > 1) return FP_EPARAM;
            h[(size_t)i] = v;
            for (int d = a.ndim - 1; d >= 0; --d) {
                if (++idx[(size_t)d] < a.shape[d]) break;
                idx[(size_t)d] = 0;
            }
        }
    }
    cudaError_t e = cudaMemcpyAsync(ws->v_side, h.data(), h.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e);
    ws->branch_on = true;
    ws->branch_tol = tol;
    ws->struct_valid = false;
    return FP_OK;
}

}  // namespace

extern "C" {

FP_API fp_status fp_prox(const fp_op *op, double gamma, const fp_array *x, fp_array *out, const fp_options *opt,
                         fp_workspace *ws, fp_info *info) {
    return guard([&] { return prox_impl(op, gamma, x, out, opt, ws, info, false, nullptr); });
}

FP_API fp_status fp_prox_steps(const fp_op *op, const fp_array *gamma, const fp_array *x, fp_array *out,
                               const fp_options *opt, fp_workspace *ws) {
    return guard([&] {
        if (!gamma) return FP_EINVAL;
        return prox_impl(op, 0.0, x, out, opt, ws, nullptr, false, gamma);
    });
}

FP_API fp_status fp_prox_conj(const fp_op *op, double sigma, const fp_array *y, fp_array *out,
                              const fp_options *opt, fp_workspace *ws, fp_info *info) {
    return guard([&] { return prox_impl(op, sigma, y, out, opt, ws, info, true, nullptr); });
}

FP_API void fp_b200_release_cached(void) { pool_release_cached(); }

FP_API fp_status fp_b200_workspace_stats(const fp_workspace *ws, int64_t *kernel_launches, int64_t *step_launches) {
    if (!ws || !ws->info_valid) return FP_EINVAL;
    if (kernel_launches) *kernel_launches = ws->kernel_launches;
    if (step_launches) *step_launches = ws->launches;
    return FP_OK;
}

FP_API fp_status fp_b200_workspace_time_steps(fp_workspace *ws, int on) {
    if (!ws) return FP_EINVAL;
    ws->time_steps = on != 0;
    return FP_OK;
}

FP_API fp_status fp_b200_vjp_images(const fp_workspace *ws, double *ggamma, double *gweights, int64_t count) {
    if (!ws || count < 0) return FP_EINVAL;
    const int64_t B = (int64_t)ws->vjp_gg_img.size();
    if (count != B || B != ws->g.B) return FP_EINVAL;
    const int64_t k = B ? (int64_t)ws->vjp_gw_img.size() / B : 0;
    for (int64_t b = 0; b < B; ++b) {
        if (ggamma) ggamma[b] = ws->vjp_gg_img[(size_t)b];
        if (gweights)
            for (int64_t a = 0; a < k; ++a) gweights[b * k + a] = ws->vjp_gw_img[(size_t)(b * k + a)];
    }
    return FP_OK;
}

FP_API fp_status fp_b200_workspace_step_times(const fp_workspace *ws, int kind, double *ms, int64_t *launches) {
    if (!ws || kind < 0 || kind > 3) return FP_EINVAL;
    if (ms) *ms = ws->tms[kind];
    if (launches) *launches = ws->tcount[kind];
    return FP_OK;
}

FP_API fp_status fp_jvp(const fp_op *op, const fp_workspace *ws, const fp_array *dx, double dgamma,
                        const fp_array *dparams, fp_array *dout) {
    return guard([&] { return jvp_impl(op, const_cast<fp_workspace *>(ws), dx, dgamma, dparams, dout); });
}

FP_API fp_status fp_vjp(const fp_op *op, const fp_workspace *ws, const fp_array *g, fp_array *gx, double *ggamma,
                        fp_array *gparams) {
    return guard([&] { return vjp_impl(op, const_cast<fp_workspace *>(ws), g, gx, ggamma, nullptr, gparams); });
}

FP_API fp_status fp_vjp_device(const fp_op *op, const fp_workspace *ws, const fp_array *g, fp_array *gx,
                               fp_array *ggamma, fp_array *gparams) {
    return guard([&] { return vjp_impl(op, const_cast<fp_workspace *>(ws), g, gx, nullptr, ggamma, gparams); });
}

FP_API fp_status fp_op_struct_kind(const fp_op *op, int *kind) {
    if (!op || !kind) return FP_EINVAL;
    // isotropic: J = M (M^T (I + G^T H G) M)^-1 M^T, range span M, not a
    // projector; anisotropic: the average over each component, a projector
    *kind = op->kind == kIso ? FP_STRUCT_CURVED : FP_STRUCT_PROJECTOR;
    return FP_OK;
}

FP_API fp_status fp_workspace_units(const fp_workspace *ws, int64_t *count, int64_t *size) {
    return guard([&] { return units_impl(ws, count, size); });
}

FP_API fp_status fp_workspace_states(const fp_workspace *ws, fp_array *state, int64_t *nfixed) {
    return guard([&] { return states_impl(const_cast<fp_workspace *>(ws), state, nfixed); });
}

FP_API fp_status fp_workspace_regions(const fp_workspace *ws, fp_array *labels, fp_array *sign, int64_t *nregions,
                                      int64_t count) {
    return guard([&] { return regions_impl(const_cast<fp_workspace *>(ws), labels, sign, nregions, count); });
}

FP_API fp_status fp_workspace_constraint(const fp_workspace *ws, fp_array *coef, int8_t *active, int64_t count) {
    return guard([&] { return constraint_impl(const_cast<fp_workspace *>(ws), coef, active, count); });
}

FP_API fp_status fp_workspace_deriv_exact(const fp_workspace *ws, int *exact, double *smoothing) {
    return guard([&] { return deriv_exact_impl(ws, exact, smoothing); });
}

FP_API fp_status fp_workspace_kinks(const fp_workspace *ws, double tol, fp_array *mask, int64_t *count) {
    return guard([&] { return kinks_impl(const_cast<fp_workspace *>(ws), tol, mask, count); });
}

FP_API fp_status fp_workspace_set_branch(fp_workspace *ws, const fp_array *side, double tol) {
    return guard([&] { return set_branch_impl(ws, side, tol); });
}

FP_API fp_status fp_workspace_refine(const fp_op *op, fp_workspace *ws, double tol, int max_iter, fp_array *out,
                                     fp_info *info) {
    return guard([&] { return refine_impl(op, ws, tol, max_iter, out, info); });
}

}  // extern "C"
