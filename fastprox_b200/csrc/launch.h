// Kernel launchers of the image-TV engine, callable from plain C++ (api.cpp).
// Every pointer is device memory owned by the workspace unless noted.
#pragma once

#include <cuda_runtime_api.h>

#include "engine.h"

namespace fpb {

// Device buffers of an isotropic solve (see engine.h for the layout).
struct IsoBuffers {
    void *d = nullptr;          // B x N of T
    void *U[2] = {nullptr, nullptr};
    void *V[2] = {nullptr, nullptr};
    void *dual = nullptr;       // k x B x N of T
    const void *alpha = nullptr;  // pixel weights (T), N or B x N, or null
    IsoImage *img = nullptr;
    IsoState *st = nullptr;
    double *gammas = nullptr;   // B steps
    double *part = nullptr;     // B x max_part x 2
    unsigned *ticket = nullptr; // B
    int *live = nullptr;        // images still iterating
    int *err = nullptr;         // set by a kernel whose copies never completed
    int max_part = 0;
    // The step's images: with lmap, launch slot z runs image lmap[z] for
    // z < *lcnt (the images still live when the list was built, in order);
    // without, slot z runs image z.
    const int *lmap = nullptr;
    const int *lcnt = nullptr;
};

// Launch shape of the step kernel, picked per geometry (and by the tuner).
struct StepShape {
    int kind = 4;   // 1: generic (one thread per pixel), 4: 2D lean row-marching, 5: 3D slice-marching tiles
    int vec = 1;    // pixels per thread along the contiguous axis (2D; 3D: 2 for the two-voxel step)
    int bx = 128;   // threads per block
    int rows = 16;  // rows per block (2D), slices per block (3D)
    int gx = 1, gy = 1;  // blocks per image = gx * gy
};

StepShape iso_pick_shape(int dtype, const Geometry &g, int rows_hint, int bx_hint, int kind_hint = 0);
int iso_setup_blocks(const Geometry &g);

// Set-up: stage x (contiguous, device) into d, per-image scans, state
// initialisation, and the warm-start projection of the stored dual.
cudaError_t iso_setup(int dtype, const Geometry &g, const IsoCall &c, const IsoBuffers &bf, const void *x,
                      int warm, int par, cudaStream_t s);
// The list of live images (by their states), for bf.lmap / bf.lcnt.
cudaError_t iso_live_list(const IsoState *st, int64_t B, int *lmap, int *lcnt, cudaStream_t s);
// One dual-FISTA iteration (and the gap / restart tests it carries) for
// every live image, reading buffers par and writing par ^ 1, over nimg launch
// slots (g.B, or at least the count of bf's live list).
// variant (the lean and 3D kernels, chosen from the iteration index k of a call):
// 1 the cold first iteration (u = v = 0), 2 a launch carrying a gap check, 0 otherwise;
// kVariantPair two plain iterations (the lean 2D shape only).
cudaError_t iso_step(int dtype, const Geometry &g, const IsoCall &c, const IsoBuffers &bf, const StepShape &sh,
                     int par, int variant, int64_t nimg, cudaStream_t s);
// Variants of iso_step running iterations k and k + 1 in one launch, where
// iso_pair_ok (the lean 2D shape over whole rows) and k + 1 < max_iter:
// kVariantPair for k = 1 mod 4 (neither has a check), kVariantPairGap for
// k = 3 mod 4 (the second carries the gap check and the restart test; when
// it passes, the final u is the first iterate, formed again by iso_redo).
constexpr int kVariantPair = 3;
constexpr int kVariantPairGap = 4;
bool iso_pair_ok(const Geometry &g, const StepShape &sh, int max_part);
inline int iso_pair_at(int64_t k, int max_iter) {
    if (k <= 0 || k + 1 >= max_iter) return -1;
    if ((k & 3) == 1) return kVariantPair;
    if ((k & 3) == 3) return kVariantPairGap;
    return -1;
}
inline int iso_variant(int64_t k, int max_iter, bool warm) {
    if (k == 0) return warm ? 2 : 1;
    return (k % 4 == 0 || k == max_iter) ? 2 : 0;
}
// Iterations k .. k + 3 in one launch (the quad), for k = 1 mod 4 and
// k + 3 < max_iter where iso_quad_ok (2D float32 rows of a multiple of 4
// pixels): the fourth carries the gap check of the third iterate and the
// restart test; when the check passes, the final u is the third iterate,
// formed again by iso_redo.
constexpr int kVariantQuad = 5;
bool iso_quad_ok(int dtype, const Geometry &g, int max_part);
// Partial-sum slots per image the quad needs (one per row and warp strip).
int64_t iso_quad_parts(const Geometry &g);
inline int iso_quad_at(int64_t k, int max_iter) {
    return (k > 0 && (k & 3) == 1 && k + 3 < max_iter) ? kVariantQuad : -1;
}
// The final u of images whose checked pair (or quad) launch passed at its
// first (third) iterate (state redo), formed again from that launch's input
// buffers; the state then points at it. Before any read of a solve's final
// dual. quads: quad launches may have run (they have their own redo launch).
cudaError_t iso_redo(int dtype, const Geometry &g, const IsoCall &c, const IsoBuffers &bf, cudaStream_t s,
                     bool quads = false);
// z = x - G^T q into out (contiguous, device, x's dtype), the dual into
// bf.dual, for every image by its mode; exact 1D TV for single-axis images.
cudaError_t iso_finalize(int dtype, const Geometry &g, const IsoCall &c, const IsoBuffers &bf, void *out,
                         cudaStream_t s);

// One step of a ragged batch over the work list of `vec` (items[0 ..
// *n_items), grid >= *n_items blocks): the single-step launch (each block in
// the variant its image asks for), then the pair variants where they apply.
cudaError_t iso_ragged_step(int dtype, int vec, const RagItem *items, const int *n_items, int grid,
                            const RagSlot *slots, const IsoCall &c, const IsoBuffers &bf, cudaStream_t s);
// Whether the ragged step on a list of `vec`-wide rows adds the two pair
// variants (float, 4-wide rows, pairs not switched off).
bool iso_ragged_pairs(int dtype, int vec);
// The ragged step's quad launch over its own work list (items[0 .. *n_items),
// an item a block of quad strips: its slot, its tile index, first row and
// first strip): four iterations for the images whose state asks for them
// (slots with nquad > 0, iteration 1 mod 4, not across max_iter); the other
// launches of the step leave those images alone.
cudaError_t iso_ragged_quad_step(const RagItem *items, const int *n_items, int grid, const RagSlot *slots,
                                 const IsoBuffers &bf, cudaStream_t s);
// Strips of a quad pass over rows of W pixels, and strips per quad block.
int iso_quad_strips(int W);
int iso_quad_warps();
bool pairs_enabled();

// Fills gammas[i] = v for i < n.
cudaError_t fill_double(double *dst, double v, int64_t n, cudaStream_t s);
// Gathers a strided array of n_dims dims into a contiguous one (element
// strides, dtype 1 = f32, 2 = f64; the destination dtype may differ: it
// converts). Used for strided inputs, outputs and per-image steps.
cudaError_t strided_copy(const void *src, int src_dtype, const int64_t *shape, const int64_t *src_strides,
                         int ndim, void *dst, int dst_dtype, const int64_t *dst_strides, cudaStream_t s);
// out = y - out (the conjugate's y - prox(y)), contiguous, n entries.
// x = d 2^e[b] for each image b of N entries (e: B ints on the device).
cudaError_t unscale_images(int dtype, const void *d, const int *e, int64_t N, int64_t B, void *x, cudaStream_t s);
cudaError_t conj_finish(int dtype, const void *y, void *out, int64_t n, cudaStream_t s);

}  // namespace fpb
