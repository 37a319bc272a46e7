// Host-visible structures of the isotropic TV derivative (tv_vjp.cu).
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>

#include "aniso.h"
#include "engine.h"

namespace fpb {

enum CgStatus : int { kCgLive = 0, kCgDone = 1 };

struct VjpGeom {
    int k;
    int64_t L[3], S[3];
    int64_t N, B;
    double wa[3];  // active axis weights (0 elsewhere)
    double wh[3];  // wa / wmax, as the forward used them
    double wmax;
    double eta;    // relative margin below the radius that counts as inside
    int act1;      // the active axis when there is exactly one, else -1
    // anisotropic structure: the largest edge weight along each axis (1
    // without edge weights), the axis weights, and the rounding allowance
    double bmax[3];
    double w[3];
    double eps_t;  // the epsilon of the iterates' dtype
    double stol;   // the tolerance of a branch override (side in VjpBuffers)
};

// A direction in the axis weights for the forward derivative.
struct JvpDir {
    double dw[3];
};

// Per image, from the kept forward (tv_iso.cpp:559-570): the step at the
// solved scale, the curvature cap, the certified relative error of z (the
// default tolerance of the conjugate gradients) and the flat threshold.
struct VjpImage {
    double gs, mu, rel, thr;
};

// Per image of an anisotropic kept point: its step (at the input's scale),
// its gap at the solved scale, and the jump thresholds of the structure
// (tv_aniso.cpp:1257-1300; tau NaN: no jump certified).
struct AnVjpImage {
    double gamma, gap, tau, tau0;
};

struct CgState {
    double rz, bn, alpha, beta, res, tol;
    int it, status, max_iter, fx;
};

struct VjpBuffers {
    // the forward's point
    const void *d = nullptr;
    const void *U[2] = {nullptr, nullptr};  // the forward's buffers, indexed by its fin_par
    const IsoImage *img = nullptr;
    const IsoState *st = nullptr;
    const void *alpha = nullptr;
    int64_t alpha_stride = 0;
    int dtype = 1;
    // structure
    uint8_t *flat = nullptr;
    int *root = nullptr, *cnt = nullptr;
    double *gz = nullptr;  // k x B x N
    unsigned long long *acc = nullptr;  // 2 x B x N, 128-bit region accumulators
    // conjugate gradients (region vectors at the roots' slots) and scratch
    double *b = nullptr, *x = nullptr, *r = nullptr, *pv = nullptr, *qv = nullptr, *dinv = nullptr, *y = nullptr;
    double *h = nullptr;  // k x B x N
    VjpImage *vimg = nullptr;
    CgState *cg = nullptr;
    double *ggam = nullptr;  // per-image step gradient
    double *gw = nullptr;    // per-image axis-weight gradients, 3 per image
    // anisotropic kept point: the solved z (z or zp per image), the dual at
    // the input's scale, edge weights, per-image solver records and the
    // structure's edge codes (2 bits per axis: 1 for +, 2 for -); S_{C,a}
    // at the roots' slots in gz
    const void *zp = nullptr;
    const void *qd = nullptr;
    const void *beta = nullptr;
    const AnImage *aimg = nullptr;
    const AnState *ast = nullptr;
    AnVjpImage *avimg = nullptr;
    uint8_t *code = nullptr;
    const int8_t *side = nullptr;  // a branch override per entry (-1, 0, +1), or null
    double *part = nullptr;
    unsigned *ticket = nullptr;
    int *live = nullptr, *err = nullptr;
    int max_part = 0;
};

cudaError_t vjp_structure(int dtype, const VjpGeom &g, const VjpBuffers &bf, cudaStream_t s);
// Anisotropic TV (tv_aniso.cpp:1012-1180, 1367-1440): the structure of the
// kept point (flat edges, components, boundary sums S_{C,a}); the VJP (gx,
// the step's gradient per image into ggam, the axis weights' into gw and,
// with edge weights, the edge weights' summed over the images into gb, k N
// doubles on the host); the JVP (dbeta: k N doubles on the device, or null).
cudaError_t an_vjp_structure(int dtype, const VjpGeom &g, const VjpBuffers &bf, cudaStream_t s);
cudaError_t an_vjp_solve(int dtype, const VjpGeom &g, const VjpBuffers &bf, const void *gin, void *gx, int conj,
                         bool params, double *gb, cudaStream_t s, int64_t *launches);
// Structure queries of a kept point whose structure is built (the reference's
// fp_workspace_regions and fp_workspace_kinks, api.cpp:1076-1170, 857-875):
// per image the labels of its regions numbered in order of their first
// entries into labels (B x N int32), their count into nreg (B doubles; -1 for
// a NaN image, whose labels are -1); the kink codes at tolerance tol into
// mask (B x N int8, zeroed here), z and the dual at the input's scale.
cudaError_t query_labels(bool aniso, const VjpGeom &g, const VjpBuffers &bf, int32_t *labels, double *nreg,
                         cudaStream_t s);
cudaError_t query_kinks(int dtype, bool aniso, const VjpGeom &g, const VjpBuffers &bf, const double *gam,
                        double tol, int8_t *mask, cudaStream_t s);
// A contiguous device array of n elements of esize bytes into a strided one
// (ndim <= 8 axes, strides in elements).
cudaError_t scatter_elements(const void *src, size_t esize, int ndim, const int64_t *shape, const int64_t *strides,
                             void *dst, cudaStream_t s);
cudaError_t an_jvp_solve(int dtype, const VjpGeom &g, const VjpBuffers &bf, const void *dx, void *dz, double dgamma,
                         const JvpDir &dir, const double *dbeta, int conj, cudaStream_t s, int64_t *launches);
// gx = J^T gin per image, the step's gradient into ggam and, with params,
// the axis weights' into gw and the pixel weights' (summed over the images)
// into qv[0, N).
cudaError_t vjp_solve(int dtype, const VjpGeom &g, const VjpBuffers &bf, const void *gin, void *gx, double tol,
                      int max_iter, int conj, bool params, cudaStream_t s, int *h_live, cudaEvent_t ev,
                      int64_t *launches);
// dz = J_x dx + (dz/dgamma) dgamma + (dz/dw) dw + (dz/dalpha) dalpha per image;
// dx and dalpha (N doubles on the device, outside x, r, y and h) may be null.
cudaError_t jvp_solve(int dtype, const VjpGeom &g, const VjpBuffers &bf, const void *dx, void *dz, double dgamma,
                      const JvpDir &dir, const double *dalpha, double tol, int max_iter, int conj, cudaStream_t s,
                      int *h_live, cudaEvent_t ev, int64_t *launches);

}  // namespace fpb
