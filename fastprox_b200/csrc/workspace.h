// The opaque fp_op and fp_workspace of the C ABI (host side).
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>
#include <vector>

#include "../../include/fastprox_b200.h"
#include "engine.h"
#include "aniso.h"
#include "launch.h"
#include "vjp.h"

namespace fpb {
enum OpKind : int { kIso = 1, kAniso = 2 };
}

// Immutable and shareable: device copies of its parameters live in the
// workspaces (the reference's fp_op, src/core/op.hpp).
struct fp_op {
    int kind = 0;                 // fpb::OpKind
    int k = 2;                    // image axes
    double w[3] = {0, 0, 0};      // axis weights
    std::vector<double> spatial;  // pixel weights (iso, N) or edge weights (aniso, k N), C order
    int64_t sshape[3] = {1, 1, 1};
    double smax = 0.0;
    bool huber = false;  // Huber-smoothed TV (fp_b200_op_tv_iso_huber / _aniso_huber), smoothing delta
    double delta = 0.0;
};

// One array shape, dtype and device; calls on it must not overlap. Every
// device byte is allocated in fp_workspace_create.
struct fp_workspace {
    const fp_op *op = nullptr;
    int device = 0;
    cudaStream_t stream = nullptr;
    int dtype = 0;
    int ndim = 0;
    int64_t shape[FP_MAX_NDIM] = {};
    fpb::Geometry g{};
    bool host_mode = false;  // created with a host `like`: host arrays staged through here
    bool keep = false;
    // device memory
    void *d = nullptr, *stage = nullptr, *dual = nullptr, *spatial = nullptr;
    void *U[2] = {nullptr, nullptr}, *V[2] = {nullptr, nullptr};
    fpb::IsoImage *img = nullptr;
    fpb::IsoState *st = nullptr;
    // anisotropic TV: per-image state, the polish's scratch, FDPG-3's scratch
    fpb::AnImage *an_img = nullptr;
    fpb::AnState *an_st = nullptr;
    void *an_scratch = nullptr;
    uint8_t *an_flag = nullptr;
    int *an_parent = nullptr, *an_cnt = nullptr;
    unsigned long long *an_sum = nullptr;
    void *an_ys = nullptr, *an_segv = nullptr, *an_wt = nullptr;  // the fibre-major passes
    int *an_segk = nullptr;
    double *gammas = nullptr;
    double *part = nullptr;
    unsigned *ticket = nullptr;
    int *lmap = nullptr, *lcnt = nullptr;  // the live images of a call, B + 1 ints
    int *live = nullptr;
    int *err = nullptr;
    int max_part = 0;
    // derivative (keep_structure workspaces): structure and conjugate gradients
    uint8_t *v_flat = nullptr, *v_code = nullptr;
    int *v_root = nullptr, *v_cnt = nullptr;
    double *v_gz = nullptr, *v_h = nullptr, *v_vec = nullptr, *v_ggam = nullptr, *v_gw = nullptr;
    unsigned long long *v_acc = nullptr;
    fpb::VjpImage *v_img = nullptr;
    fpb::CgState *v_cg = nullptr;
    fpb::VjpImage *h_vimg = nullptr;
    fpb::CgState *h_cg = nullptr;
    double *h_ggam = nullptr, *h_gw = nullptr;
    bool struct_valid = false;
    bool identity = false;  // the kept call was a conjugate at sigma = 0: J = I
    int8_t *v_side = nullptr;  // an anisotropic branch override per entry (device)
    bool branch_on = false;
    double branch_tol = 0.0;
    bool conj = false;
    // pinned host memory
    int *h_live = nullptr;
    fpb::IsoImage *h_img = nullptr;
    fpb::IsoState *h_st = nullptr;
    fpb::AnImage *h_an_img = nullptr;
    fpb::AnState *h_an_st = nullptr;
    double *h_gam = nullptr;
    void *h_stage = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    void *dev_block = nullptr, *host_block = nullptr;  // every buffer above lies in one of these
    size_t host_bytes = 0;
    // launch shape and polling
    fpb::StepShape shape_{};
    int chunk = 8;
    int64_t launches = 0;         // step launches of the last call
    int64_t kernel_launches = 0;  // all kernels of the last call
    // step-launch timing (fp_b200_workspace_time_steps): an event pair around
    // each step launch of a call, created on first use; device milliseconds and
    // launches of the last call by kind (0 single, 1 pair, 2 pair with the check)
    bool time_steps = false;
    std::vector<cudaEvent_t> tev;
    double tms[4] = {0.0, 0.0, 0.0, 0.0};
    int64_t tcount[4] = {0, 0, 0, 0};
    // small anisotropic solves: a captured chunk of rounds, replayed while the
    // call's constants, the launched images and the live list are the same
    cudaGraphExec_t an_graph = nullptr;
    fpb::AnCall an_graph_c{};
    int64_t an_graph_nimg = 0;
    const int *an_graph_lmap = nullptr;
    int64_t an_graph_launches = 0;  // kernels one replay launches
    // results of the last call
    std::vector<double> gaps, zerrs;
    std::vector<int> iters;
    fp_info info{0.0, 0, 0};
    fp_status info_status = FP_OK;
    bool info_valid = false;
    bool warm = false, seeded = false, dual_valid = false, valid = false;
    double deriv_tol = 0.0;
    int deriv_max_iter = 10000;
    // the last fp_vjp's gradients per image: the step's (B) and the axis
    // weights' (B x k), before their sums over the batch
    std::vector<double> vjp_gg_img, vjp_gw_img;
    double deriv_residual = 0.0;
    int deriv_iters = 0;
};
