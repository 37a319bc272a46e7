// Host-side view of the device solver shared by the C ABI (api.cpp) and the
// kernel launchers (*.cu). Plain structs only; no torch types.
//
// Layout in HBM (one workspace, B images of N pixels each, k image axes):
//   d          B x N        T   the staged input, rescaled by 2^-e
//   U[2], V[2] B x k x N    T   dual iterate and its extrapolation, ping-pong
//   dual       k x B x N    T   the returned dual q = u / wmax * 2^e, in the
//                               reference's (ndim, *x.shape) order
//   img        B            IsoImage   per-image constants of the solve
//   st         B            IsoState   per-image iteration state
//   part       B x P x 2    double     per-block partial sums
//   ticket     B            unsigned   last-block-done counters
#pragma once

#include <cstddef>
#include <cstdint>

namespace fpb {

enum ImgMode : int {
    kModeFdpg = 0,      // dual FISTA (two or more active axes, or pixel weights)
    kModeIdentity = 1,  // no active axis: z = x, dual 0
    kModeTv1d = 2,      // one active axis, no pixel weights: exact 1D TV
    kModeNan = 3,       // an image holding a NaN: z and dual NaN, gap NaN
    kModeInf = 4,       // an image holding +-Inf: FP_EINVAL
};

enum ImgStatus : int { kLive = 0, kConverged = 1, kNotConv = 2, kFinished = 3 };

// Per-image constants, written by the set-up kernels.
struct IsoImage {
    double gamma_in;  // the step of this image
    double radius;    // gamma wmax 2^-e (capped at bound without pixel weights)
    double bound;     // 2 imbalance / whmin + DBL_MIN
    double target;    // tol |d|^2 / 2 at the solved scale
    double dd;        // |d|^2 at the solved scale
    double mean;
    double maxabs;    // max |x| before scaling
    int e;            // the power-of-two rescaling exponent
    int mode;         // ImgMode
    int flags;        // bit 0: NaN seen, bit 1: Inf seen
    int pad;
};

// Per-image iteration state, advanced by the last block of each step launch.
// Mirrors the scalars of the reference's fdpg loop (src/ops/tv_iso.cpp:488-537).
struct IsoState {
    int it;        // iterations done
    int since;     // iterations since the last restart
    int last;      // the interval of the last restart
    int status;    // ImgStatus
    int vsel;      // 1: the next step reads v = u (a restart fired)
    int zero_in;   // 1: u = v = 0 (cold start, nothing staged)
    int warm;      // 1: the gap is checked before the first iteration
    int fin_par;   // buffer parity holding the final u
    int redo;      // the final u is redo more iterations from the buffers of fin_par, reading v = u when
                   // redo_vsel: 1 (a checked pair's check passed at its first iterate, which it did not
                   // store) or 3 (a quad's check passed at its third iterate); 0 otherwise
    int redo_vsel;
    double tn;     // fista_t(t) of the next iteration, t its momentum scalar
    double beta;   // (t - 1) / tn of the next iteration
    double gp;     // last gap checked
    double dot;    // last restart dot product
    double redo_tn, redo_beta;  // tn and beta of the first iteration redone (redo = 3)
};

struct Geometry {
    int k;            // 2 or 3 image axes
    int64_t L[3];     // extents (axis 0 slowest)
    int64_t N;        // pixels per image
    int64_t B;        // images
};

// Per-call constants of an isotropic solve.
struct IsoCall {
    double wh[3];     // w / wmax on active axes, 0 elsewhere
    double wmax;
    double whmin;
    double tau;       // 1 / (4 sum wh^2)
    double tol;
    int max_iter;
    int has_alpha;
    int64_t alpha_stride;  // 0: one map for the batch; N: one per image
    double alpha_max;
    double step_scale;     // max w * max alpha (the operator's step_scale)
    int na;                // active axes (the same for every image of gamma > 0)
    int act_axis;          // the active axis when na == 1
    double w_act;          // its weight
    int huber;             // Huber-smoothed TV: 0 none, 1 isotropic, 2 anisotropic (per axis component)
    double delta;          // its smoothing delta (at the input's scale)
};

// One image of a ragged batch: its shape, its place in the arena (pixel
// offset; the dual pairs sit at twice it), its tiles and its stopping limit.
struct RagSlot {
    int H, W;
    int64_t off;
    int nblk;       // tiles (blocks) of the image
    int max_iter;
    int rows;       // rows per tile
    int vec;        // pixels per thread along a row
    double wh0, wh1, tau;
    int nquad;      // tiles of the quad launch (0: the image takes no quads)
    int qrows;      // rows per quad tile
};

// One tile of the work list: the image's slot, the tile's index within the
// image (its partial-sum slot), its first row and first column.
struct RagItem {
    int slot, blk, r0, cs;
};

}  // namespace fpb
