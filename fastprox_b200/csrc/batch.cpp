// The ragged batch engine: isotropic 2D TV on images of mixed sizes in one
// set of launches, with images admitted and retired between steps
// (continuous batching). A B200 extension of the C ABI; no counterpart in the
// reference, whose driver takes one array shape per call.
//
// Device memory (all allocated at creation): an arena of pixels holding d and
// the ping-pong dual pairs u, v of every admitted image (a first-fit free list
// of pixel ranges on the host places them), per-slot constants and state,
// partial sums and tickets, and two work lists of (image, tile) items, one
// for rows of a multiple of 4 pixels (16-byte vectors) and one for the rest.
// A step launches the single-step kernel over each list (each block in the
// variant its image's state asks for), on the 4-wide float list the two pair
// variants (two iterations per launch), and over a third list of quad tiles
// (float rows of a multiple of 4 pixels) the quad (four iterations per
// launch); chunks of steps are replayed as CUDA graphs, captured again only
// when the work lists outgrow their current size class.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <vector>

#include "../../include/fastprox_b200.h"
#include "engine.h"
#include "launch.h"
#include "workspace.h"

using namespace fpb;

namespace {

struct Range {
    int64_t start, len;
};

struct SlotHost {
    bool used = false;
    int H = 0, W = 0;
    int64_t off = 0, len = 0;
    void *out = nullptr;  // the caller's z (device)
    int first_item = 0, n_items = 0, vec = 1;
    bool quad = false;  // the slot may take quad launches (its redo)
};

template <class F>
fp_status guard_b(F &&f) noexcept {
    try {
        return f();
    } catch (const std::bad_alloc &) {
        return FP_ENOMEM;
    } catch (...) {
        return FP_EINTERNAL;
    }
}

}  // namespace

struct fp_b200_batch {
    const fp_op *op = nullptr;
    int device = 0;
    cudaStream_t stream = nullptr;
    int dtype = FP_F32;
    int64_t max_slots = 0, max_pixels = 0, max_items = 0;
    int max_part = 4096;
    // device
    void *d = nullptr, *U[2] = {nullptr, nullptr}, *V[2] = {nullptr, nullptr}, *dual = nullptr;
    IsoImage *img = nullptr;
    IsoState *st = nullptr;
    double *gammas = nullptr, *part = nullptr;
    unsigned *ticket = nullptr;
    int *live = nullptr, *err = nullptr;
    RagSlot *slots = nullptr;
    RagItem *items[3] = {nullptr, nullptr, nullptr};  // [0] vec 4 (or 2 for double), [1] vec 1, [2] quad tiles
    int *n_items = nullptr;                           // 3 counts
    std::vector<void *> allocs, pinned;
    // host
    std::vector<Range> free_list;
    std::vector<SlotHost> sh;
    RagSlot *h_slots = nullptr;
    RagItem *h_items[3] = {nullptr, nullptr, nullptr};
    int *h_n = nullptr;
    IsoState *h_st = nullptr;
    IsoImage *h_img = nullptr;
    int *h_live = nullptr;
    bool items_dirty = true;
    int grid[3] = {0, 0, 0};
    // graphs of `chunk` steps, keyed by (grid0, grid1, grid2, chunk)
    std::map<std::tuple<int, int, int, int>, cudaGraphExec_t> graphs;
    int rows_hint = 0;
    bool quads = true;  // quad tiles for the float rows of a multiple of 4 pixels (admitted from now on)
    int quad_rows = 32;
    bool use_graphs = true;
    int64_t steps_run = 0, kernel_launches = 0;
    double wh[2] = {1.0, 1.0}, tau = 0.125;
};

namespace {

fp_status balloc(fp_b200_batch *bt, void **p, size_t bytes) {
    if (cudaMalloc(p, bytes ? bytes : 16) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return FP_ENOMEM;
    }
    bt->allocs.push_back(*p);
    return FP_OK;
}

fp_status halloc(fp_b200_batch *bt, void **p, size_t bytes) {
    if (cudaHostAlloc(p, bytes ? bytes : 16, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return FP_ENOMEM;
    }
    bt->pinned.push_back(*p);
    return FP_OK;
}

void release(fp_b200_batch *bt) {
    for (auto &kv : bt->graphs) cudaGraphExecDestroy(kv.second);
    bt->graphs.clear();
    for (void *p : bt->allocs) cudaFree(p);
    for (void *p : bt->pinned) cudaFreeHost(p);
    bt->allocs.clear();
    bt->pinned.clear();
}

// first fit in the free list; len is rounded to 4 pixels (16-byte bases)
bool arena_take(fp_b200_batch *bt, int64_t len, int64_t &off) {
    len = (len + 3) / 4 * 4;
    for (size_t i = 0; i < bt->free_list.size(); ++i) {
        Range &r = bt->free_list[i];
        if (r.len >= len) {
            off = r.start;
            r.start += len;
            r.len -= len;
            if (r.len == 0) bt->free_list.erase(bt->free_list.begin() + (long)i);
            return true;
        }
    }
    return false;
}

void arena_give(fp_b200_batch *bt, int64_t off, int64_t len) {
    len = (len + 3) / 4 * 4;
    bt->free_list.push_back({off, len});
    std::sort(bt->free_list.begin(), bt->free_list.end(), [](const Range &a, const Range &b) { return a.start < b.start; });
    std::vector<Range> merged;
    for (const Range &r : bt->free_list) {
        if (!merged.empty() && merged.back().start + merged.back().len == r.start) merged.back().len += r.len;
        else merged.push_back(r);
    }
    bt->free_list.swap(merged);
}

IsoBuffers buffers(fp_b200_batch *bt) {
    IsoBuffers bf;
    bf.d = bt->d;
    for (int i = 0; i < 2; ++i) {
        bf.U[i] = bt->U[i];
        bf.V[i] = bt->V[i];
    }
    bf.dual = bt->dual;
    bf.alpha = nullptr;
    bf.img = bt->img;
    bf.st = bt->st;
    bf.gammas = bt->gammas;
    bf.part = bt->part;
    bf.ticket = bt->ticket;
    bf.live = bt->live;
    bf.err = bt->err;
    bf.max_part = bt->max_part;
    return bf;
}

// the buffers of one slot as a batch of one image (set-up, finalisation)
IsoBuffers slot_buffers(fp_b200_batch *bt, int slot) {
    const size_t T = bt->dtype == FP_F32 ? 4 : 8;
    const SlotHost &s = bt->sh[(size_t)slot];
    IsoBuffers bf = buffers(bt);
    bf.d = static_cast<char *>(bt->d) + (size_t)s.off * T;
    for (int i = 0; i < 2; ++i) {
        bf.U[i] = static_cast<char *>(bt->U[i]) + 2 * (size_t)s.off * T;
        bf.V[i] = static_cast<char *>(bt->V[i]) + 2 * (size_t)s.off * T;
    }
    bf.dual = static_cast<char *>(bt->dual) + 2 * (size_t)s.off * T;
    bf.img = bt->img + slot;
    bf.st = bt->st + slot;
    bf.gammas = bt->gammas + slot;
    bf.part = bt->part + (int64_t)slot * bt->max_part * 2;
    bf.ticket = bt->ticket + slot;
    return bf;
}

IsoCall call_for(fp_b200_batch *bt, const SlotHost &s, double tol, int max_iter) {
    IsoCall c{};
    const fp_op *op = bt->op;
    const int64_t L[2] = {s.H, s.W};
    double wmax_all = 0.0;
    for (int a = 0; a < 2; ++a)
        if (L[a] > 1) wmax_all = std::max(wmax_all, op->w[a]);
    double wa[2] = {0.0, 0.0};
    int na = 0, act = 0;
    for (int a = 0; a < 2; ++a)
        if (op->w[a] > 0.0 && L[a] > 1 && op->w[a] >= 1e-100 * wmax_all) {
            wa[a] = op->w[a];
            ++na;
            act = a;
        }
    double wmax = std::max(wa[0], wa[1]);
    c.na = na;
    c.act_axis = act;
    c.w_act = op->w[act];
    c.wmax = wmax > 0.0 ? wmax : 1.0;
    double whmin = 1.0, L2 = 0.0;
    for (int a = 0; a < 3; ++a) {
        c.wh[a] = (a < 2 && wa[a] != 0.0) ? wa[a] / c.wmax : 0.0;
        if (a < 2 && wa[a] != 0.0) whmin = std::min(whmin, c.wh[a]);
        L2 += 4.0 * c.wh[a] * c.wh[a];
    }
    c.whmin = whmin;
    c.tau = L2 > 0.0 ? 1.0 / L2 : 0.0;
    c.tol = tol;
    c.max_iter = max_iter;
    c.has_alpha = 0;
    c.step_scale = std::max(op->w[0], op->w[1]);
    return c;
}

// the work lists from the slots in use
void rebuild_items(fp_b200_batch *bt) {
    int n[3] = {0, 0, 0};
    const int vfull = bt->dtype == FP_F32 ? 4 : 2;
    for (size_t i = 0; i < bt->sh.size(); ++i) {
        SlotHost &s = bt->sh[i];
        if (!s.used) continue;
        const int list = s.vec == vfull ? 0 : 1;
        const int span = 128 * s.vec;
        const RagSlot &rs = bt->h_slots[i];
        int blk = 0;
        for (int r0 = 0; r0 < s.H; r0 += rs.rows)
            for (int cs = 0; cs < s.W; cs += span) {
                if (n[list] < bt->max_items) bt->h_items[list][n[list]++] = RagItem{(int)i, blk, r0, cs};
                ++blk;
            }
        if (rs.nquad > 0) {  // quad tiles: qrows rows x iso_quad_warps() strips
            const int ns = iso_quad_strips(s.W), qw = iso_quad_warps();
            int qb = 0;
            for (int r0 = 0; r0 < s.H; r0 += rs.qrows)
                for (int st0 = 0; st0 < ns; st0 += qw) {
                    if (n[2] < bt->max_items) bt->h_items[2][n[2]++] = RagItem{(int)i, qb, r0, st0};
                    ++qb;
                }
        }
    }
    bt->h_n[0] = n[0];
    bt->h_n[1] = n[1];
    bt->h_n[2] = n[2];
    for (int l = 0; l < 3; ++l) {
        // a size class (a power of two) keeps captured graphs valid while the lists change within it
        int gcls = 0;
        if (n[l] > 0) {
            gcls = 256;
            while (gcls < n[l]) gcls *= 2;
        }
        bt->grid[l] = gcls;
        if (n[l]) cudaMemcpyAsync(bt->items[l], bt->h_items[l], (size_t)n[l] * sizeof(RagItem), cudaMemcpyHostToDevice,
                                  bt->stream);
    }
    cudaMemcpyAsync(bt->n_items, bt->h_n, 3 * sizeof(int), cudaMemcpyHostToDevice, bt->stream);
    bt->items_dirty = false;
}

cudaError_t launch_steps(fp_b200_batch *bt, int steps) {
    const IsoBuffers bf = buffers(bt);
    IsoCall c{};
    c.has_alpha = 0;
    const int vfull = bt->dtype == FP_F32 ? 4 : 2;
    for (int k = 0; k < steps; ++k) {
        cudaError_t e = iso_ragged_step(bt->dtype, vfull, bt->items[0], bt->n_items, bt->grid[0], bt->slots, c, bf,
                                        bt->stream);
        if (e == cudaSuccess)
            e = iso_ragged_step(bt->dtype, 1, bt->items[1], bt->n_items + 1, bt->grid[1], bt->slots, c, bf, bt->stream);
        if (e == cudaSuccess)
            e = iso_ragged_quad_step(bt->items[2], bt->n_items + 2, bt->grid[2], bt->slots, bf, bt->stream);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// kernels one step launches: the single steps on each non-empty list, the
// two pair variants on the 4-wide float list
int launches_per_step(const fp_b200_batch *bt) {
    int n = 0;
    if (bt->grid[0] > 0) n += 1 + (iso_ragged_pairs(bt->dtype, 4) ? 2 : 0);
    if (bt->grid[1] > 0) n += 1;
    if (bt->grid[2] > 0) n += 1;
    return n;
}

void trace(const char *what, cudaError_t e) {
    if (e != cudaSuccess && std::getenv("FASTPROX_B200_DEBUG"))
        std::fprintf(stderr, "fastprox_b200 batch: %s: %s\n", what, cudaGetErrorString(e));
}

cudaError_t run_chunk(fp_b200_batch *bt, int steps) {
    if (!bt->use_graphs) return launch_steps(bt, steps);
    const auto key = std::make_tuple(bt->grid[0], bt->grid[1], bt->grid[2], steps);
    auto it = bt->graphs.find(key);
    if (it == bt->graphs.end()) {
        cudaGraph_t graph = nullptr;
        cudaStream_t cap = nullptr;
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) return cudaErrorUnknown;
        cudaStream_t keep = bt->stream;
        bt->stream = cap;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            e = launch_steps(bt, steps);
            cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
            if (e == cudaSuccess) e = e2;
        }
        bt->stream = keep;
        cudaStreamDestroy(cap);
        if (e != cudaSuccess) {
            // a capture can fail while other threads use the device; run the
            // chunk as plain launches instead, and stop capturing
            trace("graph capture", e);
            cudaGetLastError();
            if (graph) cudaGraphDestroy(graph);
            bt->use_graphs = false;
            return launch_steps(bt, steps);
        }
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            trace("graph instantiate", e);
            cudaGetLastError();
            bt->use_graphs = false;
            return launch_steps(bt, steps);
        }
        it = bt->graphs.emplace(key, exec).first;
    }
    return cudaGraphLaunch(it->second, bt->stream);
}

}  // namespace

extern "C" {

FP_API fp_status fp_b200_batch_create(const fp_op *op, int64_t max_images, int64_t max_pixels, int dtype,
                                      fp_b200_batch **out) {
    return guard_b([&] {
        if (!out) return FP_EINVAL;
        *out = nullptr;
        if (!op || op->kind != kIso || op->k != 2 || !op->spatial.empty()) return FP_EINVAL;
        if (dtype != FP_F32 && dtype != FP_F64) return FP_EDTYPE;
        if (max_images < 1 || max_pixels < 1 || max_images > (1 << 20)) return FP_ESHAPE;
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            return FP_EDEVICE;
        }
        auto bt = std::make_unique<fp_b200_batch>();
        bt->op = op;
        cudaGetDevice(&bt->device);
        bt->dtype = dtype;
        bt->max_slots = max_images;
        bt->max_pixels = (max_pixels + 3) / 4 * 4 + 4 * max_images;
        // tiles: at least one per 128 x 4 x 4 pixels of the arena, plus one row of tiles per image
        bt->max_items = bt->max_pixels / 1024 + 64 * max_images + 1024;
        const size_t T = dtype == FP_F32 ? 4 : 8, P = (size_t)bt->max_pixels, S = (size_t)max_images;
        fp_status s = FP_OK;
        auto A = [&](void **p, size_t bytes) {
            if (s == FP_OK) s = balloc(bt.get(), p, bytes);
        };
        auto Hh = [&](void **p, size_t bytes) {
            if (s == FP_OK) s = halloc(bt.get(), p, bytes);
        };
        A(&bt->d, P * T);
        for (int i = 0; i < 2; ++i) {
            A(&bt->U[i], 2 * P * T);
            A(&bt->V[i], 2 * P * T);
        }
        A(&bt->dual, 2 * P * T);
        A((void **)&bt->img, S * sizeof(IsoImage));
        A((void **)&bt->st, S * sizeof(IsoState));
        A((void **)&bt->gammas, S * sizeof(double));
        A((void **)&bt->part, S * (size_t)bt->max_part * 2 * sizeof(double));
        A((void **)&bt->ticket, S * sizeof(unsigned));
        A((void **)&bt->live, 16);
        A((void **)&bt->err, 16);
        A((void **)&bt->slots, S * sizeof(RagSlot));
        A((void **)&bt->items[0], (size_t)bt->max_items * sizeof(RagItem));
        A((void **)&bt->items[1], (size_t)bt->max_items * sizeof(RagItem));
        A((void **)&bt->items[2], (size_t)bt->max_items * sizeof(RagItem));
        A((void **)&bt->n_items, 16);
        Hh((void **)&bt->h_slots, S * sizeof(RagSlot));
        Hh((void **)&bt->h_items[0], (size_t)bt->max_items * sizeof(RagItem));
        Hh((void **)&bt->h_items[1], (size_t)bt->max_items * sizeof(RagItem));
        Hh((void **)&bt->h_items[2], (size_t)bt->max_items * sizeof(RagItem));
        Hh((void **)&bt->h_n, 16);
        Hh((void **)&bt->h_st, S * sizeof(IsoState));
        Hh((void **)&bt->h_img, S * sizeof(IsoImage));
        Hh((void **)&bt->h_live, 16);
        if (s == FP_OK) {
            if (cudaMemset(bt->ticket, 0, S * sizeof(unsigned)) != cudaSuccess ||
                cudaMemset(bt->live, 0, 16) != cudaSuccess || cudaMemset(bt->err, 0, 16) != cudaSuccess ||
                cudaMemset(bt->n_items, 0, 16) != cudaSuccess || cudaMemset(bt->st, 0, S * sizeof(IsoState)) != cudaSuccess)
                s = FP_EDEVICE;
            // no slot live: every state's status is not kLive (kFinished = 3)
            std::vector<IsoState> init(S);
            for (auto &x : init) {
                std::memset(&x, 0, sizeof x);
                x.status = kFinished;
            }
            if (s == FP_OK && cudaMemcpy(bt->st, init.data(), S * sizeof(IsoState), cudaMemcpyHostToDevice) != cudaSuccess)
                s = FP_EDEVICE;
        }
        if (s != FP_OK) {
            release(bt.get());
            return s;
        }
        bt->free_list.push_back({0, bt->max_pixels});
        bt->sh.resize(S);
        if (const char *v = std::getenv("FASTPROX_B200_ROWS")) bt->rows_hint = std::atoi(v);
        *out = bt.release();
        return FP_OK;
    });
}

FP_API void fp_b200_batch_free(fp_b200_batch *bt) {
    if (!bt) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(bt->device);
    cudaStreamSynchronize(bt->stream);
    release(bt);
    cudaSetDevice(cur);
    delete bt;
}

FP_API fp_status fp_b200_batch_set_stream(fp_b200_batch *bt, void *stream) {
    if (!bt) return FP_EINVAL;
    bt->stream = static_cast<cudaStream_t>(stream);
    return FP_OK;
}

FP_API fp_status fp_b200_batch_set_graphs(fp_b200_batch *bt, int on) {
    if (!bt) return FP_EINVAL;
    bt->use_graphs = on != 0;
    return FP_OK;
}

FP_API fp_status fp_b200_batch_set_quads(fp_b200_batch *bt, int on, int rows) {
    if (!bt || rows < 0 || rows > 1024) return FP_EINVAL;
    bt->quads = on != 0;
    if (rows > 0) bt->quad_rows = rows;
    return FP_OK;
}

FP_API fp_status fp_b200_batch_set_rows(fp_b200_batch *bt, int rows) {
    if (!bt || rows < 0 || rows > 1024) return FP_EINVAL;
    bt->rows_hint = rows;
    return FP_OK;
}

FP_API fp_status fp_b200_batch_admit(fp_b200_batch *bt, const void *x, int64_t height, int64_t width, double gamma,
                                     double tol, int max_iter, void *z, int *slot_out) {
    return guard_b([&] {
        if (!bt || !x || !z || !slot_out) return FP_EINVAL;
        if (height < 1 || width < 1 || height * width >= 2147483647LL || height > (1 << 30) || width > (1 << 30))
            return FP_ESHAPE;
        if (!std::isfinite(gamma) || gamma < 0.0 || !(gamma <= 0x1p960)) return FP_EPARAM;
        if (!(tol >= 0.0) || !std::isfinite(tol) || max_iter < 1) return FP_EPARAM;
        int slot = -1;
        for (size_t i = 0; i < bt->sh.size(); ++i)
            if (!bt->sh[i].used) {
                slot = (int)i;
                break;
            }
        if (slot < 0) return FP_ENOMEM;
        const int64_t N = height * width;
        int64_t off = 0;
        if (!arena_take(bt, N, off)) return FP_ENOMEM;
        const int vfull = bt->dtype == FP_F32 ? 4 : 2;
        SlotHost &s = bt->sh[(size_t)slot];
        s.used = true;
        s.H = (int)height;
        s.W = (int)width;
        s.off = off;
        s.len = N;
        s.out = z;
        s.vec = width % vfull == 0 ? vfull : 1;
        const IsoCall c = call_for(bt, s, tol, max_iter);
        RagSlot rs{};
        rs.H = s.H;
        rs.W = s.W;
        rs.off = off;
        rs.rows = bt->rows_hint > 0 ? bt->rows_hint : (int)std::max<int64_t>(4, std::min<int64_t>(16, height / 32));
        const int span = 128 * s.vec;
        rs.nblk = (int)(((height + rs.rows - 1) / rs.rows) * ((width + span - 1) / span));
        if (rs.nblk > bt->max_part) {
            rs.rows = (int)((height + (bt->max_part / ((width + span - 1) / span)) - 1) /
                            (bt->max_part / ((width + span - 1) / span)));
            rs.nblk = (int)(((height + rs.rows - 1) / rs.rows) * ((width + span - 1) / span));
        }
        rs.max_iter = max_iter;
        rs.vec = s.vec;
        // quad tiles: float rows of a multiple of 4 pixels, two rows or more
        rs.qrows = bt->quad_rows;
        rs.nquad = 0;
        if (bt->quads && iso_ragged_pairs(bt->dtype, s.vec) && width % 4 == 0 && height >= 2) {
            const int64_t nq = ((height + rs.qrows - 1) / rs.qrows) *
                               ((iso_quad_strips((int)width) + iso_quad_warps() - 1) / iso_quad_warps());
            if (nq <= bt->max_part) rs.nquad = (int)nq;
        }
        s.quad = rs.nquad > 0;
        rs.wh0 = c.wh[0];
        rs.wh1 = c.wh[1];
        rs.tau = c.tau;
        bt->h_slots[slot] = rs;
        cudaStream_t st = bt->stream;
        const size_t T = bt->dtype == FP_F32 ? 4 : 8;
        cudaError_t e = cudaMemcpyAsync(bt->slots + slot, bt->h_slots + slot, sizeof(RagSlot), cudaMemcpyHostToDevice, st);
        IsoBuffers bf = slot_buffers(bt, slot);
        Geometry g{};
        g.k = 2;
        g.L[0] = height;
        g.L[1] = width;
        g.L[2] = 1;
        g.N = N;
        g.B = 1;
        if (e == cudaSuccess) e = cudaMemsetAsync(bt->ticket + slot, 0, sizeof(unsigned), st);
        if (e == cudaSuccess) e = fill_double(bf.gammas, gamma, 1, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(bf.d, x, (size_t)N * T, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = iso_setup(bt->dtype, g, c, bf, bf.d, 0, 0, st);
        if (e != cudaSuccess) {
            s.used = false;
            arena_give(bt, off, N);
            return e == cudaErrorMemoryAllocation ? FP_ENOMEM : FP_EDEVICE;
        }
        bt->kernel_launches += 4;
        bt->items_dirty = true;
        *slot_out = slot;
        return FP_OK;
    });
}

// Runs chunks of `steps` iterations until at least one admitted image has
// finished, none is live or max_chunks (> 0) chunks ran, finalises the
// finished ones into their z, frees their slots, and reports them (slots,
// gaps, iterations; each array max_images long). *nfinished = 0 with
// *nlive = 0: nothing was admitted.
FP_API fp_status fp_b200_batch_run(fp_b200_batch *bt, int steps, int max_chunks, int *finished, double *gaps,
                                   int *iters, int *nfinished, int *nlive) {
    return guard_b([&] {
        if (!bt || steps < 1 || !nfinished) return FP_EINVAL;
        *nfinished = 0;
        cudaStream_t st = bt->stream;
        if (bt->items_dirty) {
            // the live count from the set-ups (images that finished at set-up are not live)
            rebuild_items(bt);
        }
        const size_t S = (size_t)bt->max_slots;
        std::vector<int> done;
        const int chunks = max_chunks > 0 ? max_chunks : (1 << 20);
        for (int chunk = 0; chunk < chunks; ++chunk) {
            cudaError_t e = run_chunk(bt, steps);
            trace("run", e);
            if (e != cudaSuccess) return FP_EDEVICE;
            bt->steps_run += steps;
            bt->kernel_launches += (int64_t)steps * launches_per_step(bt);
            e = cudaMemcpyAsync(bt->h_st, bt->st, S * sizeof(IsoState), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(bt->h_live, bt->live, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            trace("poll", e);
            if (e != cudaSuccess) return FP_EDEVICE;
            for (size_t i = 0; i < S; ++i)
                if (bt->sh[i].used && bt->h_st[i].status != kLive) done.push_back((int)i);
            if (!done.empty() || *bt->h_live == 0) break;
        }
        if (nlive) *nlive = *bt->h_live;
        if (done.empty()) return FP_OK;
        // finalise: z into the caller's array, results, slot freed
        cudaError_t e = cudaSuccess;
        for (int slot : done) {
            SlotHost &s = bt->sh[(size_t)slot];
            const IsoCall c = call_for(bt, s, 0.0, bt->h_slots[slot].max_iter);
            Geometry g{};
            g.k = 2;
            g.L[0] = s.H;
            g.L[1] = s.W;
            g.L[2] = 1;
            g.N = (int64_t)s.H * s.W;
            g.B = 1;
            IsoBuffers bf = slot_buffers(bt, slot);
            if (e == cudaSuccess) e = iso_redo(bt->dtype, g, c, bf, st, s.quad);
            if (e == cudaSuccess) e = iso_finalize(bt->dtype, g, c, bf, s.out, st);
            bt->kernel_launches += 3;
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(bt->h_img, bt->img, S * sizeof(IsoImage), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return FP_EDEVICE;
        int n = 0;
        for (int slot : done) {
            SlotHost &s = bt->sh[(size_t)slot];
            const IsoImage &im = bt->h_img[slot];
            const IsoState &ss = bt->h_st[slot];
            double gap = 0.0;
            int it = 0;
            if (im.mode == kModeFdpg) {
                gap = std::ldexp(std::max(ss.gp, 0.0), 2 * im.e);
                it = ss.it;
            } else if (im.mode == kModeNan) {
                gap = NAN;
            }
            if (finished) finished[n] = slot;
            if (gaps) gaps[n] = gap;
            if (iters) iters[n] = im.mode == kModeFdpg && ss.status != kConverged ? -it : it;
            ++n;
            s.used = false;
            arena_give(bt, s.off, s.len);
            // the slot's state reads as not live until it is admitted again
            IsoState idle{};
            idle.status = kFinished;
            bt->h_st[slot] = idle;
            cudaMemcpyAsync(bt->st + slot, bt->h_st + slot, sizeof(IsoState), cudaMemcpyHostToDevice, st);
        }
        *nfinished = n;
        bt->items_dirty = true;
        return FP_OK;
    });
}

FP_API fp_status fp_b200_batch_stats(const fp_b200_batch *bt, int64_t *kernel_launches, int64_t *steps,
                                     int64_t *free_pixels) {
    if (!bt) return FP_EINVAL;
    if (kernel_launches) *kernel_launches = bt->kernel_launches;
    if (steps) *steps = bt->steps_run;
    if (free_pixels) {
        int64_t f = 0;
        for (const Range &r : bt->free_list) f += r.len;
        *free_pixels = f;
    }
    return FP_OK;
}

}  // extern "C"
