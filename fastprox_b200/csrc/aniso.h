// Host-visible structures of the anisotropic engine (tv_aniso.cu).
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>

namespace fpb {

enum AnMode : int { kAnAdbpg = 0, kAnFdpg3 = 1, kAnSingle = 2, kAnIdentity = 3, kAnNan = 4, kAnInf = 5 };
// kStWarm: a warm start's pass z = prox_{g1}(d + y) and its dual before the
// second check (tv_aniso.cpp:467-486)
enum AnStage : int { kStIter = 0, kStCheck = 1, kStPolish = 2, kStFinal = 3, kStDone = 4, kStWarm = 5 };

struct AnGeom {
    int k;
    int64_t L[3];
    int64_t S[3];
    int64_t N, B;
};

struct AnCall {
    double w[3];
    double tol;
    int max_iter;
    double step_scale;
    int has_beta;
    double beta_max;
    int64_t N;
    int has_adbpg, has_fdpg3;
    int warm;  // the call starts from the dual in bf.dual
};

struct AnImage {
    double gamma_in;
    double lam[3];   // gamma w_a 2^-e on active axes, else 0
    double target;   // tol |d|^2 / 2 at the solved scale
    double dd;
    double maxabs;
    int e, mode, flags, na, a1, a2, fx_shift, pad;
};

// The scalars of TVAniso::adbpg / fdpg3 (src/ops/tv_aniso.cpp:429-616).
struct AnState {
    int status, stage, it, since, last, restart, warm, polished, zsel, pol_accept;
    int chk_next, chk_prev_it;
    int wphase, pad;  // a warm start: 1 before its first check's outcome, 2 before its second's, else 0
    double tn, beta, gp, gz, accept, chk_prev, pol_next;
};

struct AnBuffers {
    void *d = nullptr, *z = nullptr, *u = nullptr, *y = nullptr, *wv = nullptr, *zp = nullptr, *scratch = nullptr;
    void *dual = nullptr;
    const void *beta = nullptr;  // edge weights (T), k x N, or null
    uint8_t *flag = nullptr;
    int *parent = nullptr;
    unsigned long long *sum = nullptr;
    int *cnt = nullptr;
    AnImage *img = nullptr;
    AnState *st = nullptr;
    double *gammas = nullptr;
    double *part = nullptr;
    unsigned *ticket = nullptr;
    int *live = nullptr;
    int *err = nullptr;
    int max_part = 0;
    // a round's images: with lmap, launch slot z runs image lmap[z] for z < *lcnt
    const int *lmap = nullptr;
    const int *lcnt = nullptr;
    // the fibre-major passes: y of a pass's fibres (B x N), the segment ends of
    // their scans (value, first entry), the edge weights of strided axes (k x N)
    void *ys = nullptr, *segv = nullptr;
    int *segk = nullptr;
    const void *wt = nullptr;
};

// CheckSchedule::done (src/ops/tv_aniso.cpp:400-413): after the first two
// checks, every 4 iterations, sooner when the rate of the gap's fall
// predicts the target.
#ifdef __CUDACC__
__device__ __forceinline__ void check_done(AnState &s, double gp, double target) {
    int step = 1;
    if (s.chk_prev_it >= 0) {
        step = 4;
        if (gp < s.chk_prev && gp > target) {
            const double n = log(target / gp) / log(gp / s.chk_prev) * (double)(s.it - s.chk_prev_it);
            if (n < 4.0) step = n > 1.0 ? (int)n : 1;
        }
    }
    s.chk_prev_it = s.it;
    s.chk_prev = gp;
    s.chk_next = s.it + step;
}
#endif

int an_pixel_blocks(const AnGeom &g);
// Whether rounds run the fibre-major passes (FASTPROX_B200_AN_FIB=0: the tiled ones).
bool aniso_fm_enabled();
// The edge weights beta (k x N of the dtype) of every strided axis into wt,
// fibre-major (entry i of fibre f of axis a at a N + f L_a + i).
cudaError_t aniso_weights_fm(int dtype, const AnGeom &g, const void *beta, void *wt, cudaStream_t s);
cudaError_t aniso_setup(int dtype, const AnGeom &g, const AnCall &c, const AnBuffers &bf, const void *x,
                        cudaStream_t s);
// A warm start (tv_aniso.cpp:316-320, 436-486, 539-543, 630-684): the dual
// in bf.dual (the input's scale) made feasible fibre by fibre at the solved
// scale, y and the extrapolation from it, and z = d - sum_a q_a for a first
// check at iteration 0.
cudaError_t aniso_warm(int dtype, const AnGeom &g, const AnCall &c, const AnBuffers &bf, cudaStream_t s);
// Kernel attributes the rounds need, set before the first capture or launch.
void aniso_prepare(int dtype);
// One round over nimg launch slots (g.B, or at least the count of bf's live list).
cudaError_t aniso_round(int dtype, const AnGeom &g, const AnCall &c, const AnBuffers &bf, int64_t nimg,
                        cudaStream_t s, int64_t *launches);
// The list of live images (by their states), for bf.lmap / bf.lcnt.
cudaError_t aniso_live_list(const AnState *st, int64_t B, int *lmap, int *lcnt, cudaStream_t s);
cudaError_t aniso_output(int dtype, const AnGeom &g, const AnBuffers &bf, void *out, cudaStream_t s);

}  // namespace fpb
