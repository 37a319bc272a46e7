/* A C program of the reference's users: written against the reference's
 * public header (include/fastprox.h, ABI v1) and linked to
 * libfastprox_b200.so instead of libfastprox. It builds the image-TV
 * operators, reads their parameters, creates a workspace for a small host
 * batch and solves it: FP_OK or FP_ENOTCONV where a CUDA device is present,
 * FP_EDEVICE without one (this library has no CPU solver). Prints one line per
 * check; exits non-zero on a mismatch. */
#include <stdio.h>
#include <string.h>

/* the reference's header, or this library's (FP_HEADER on the command line) */
#include FP_HEADER

#define CHECK(c)                                                  \
    do {                                                          \
        if (!(c)) {                                               \
            printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c);    \
            return 1;                                             \
        }                                                         \
    } while (0)

int main(int argc, char **argv) {
    int gpu = argc > 1 && strcmp(argv[1], "gpu") == 0;
    CHECK(fp_abi_version() == FP_ABI_VERSION);
    printf("version %s\n", fp_version_string());
    fp_options opt;
    fp_options_init(&opt);
    CHECK(opt.max_iter == 1000 && opt.tol == 1e-6);
    fp_op *iso = NULL, *aniso = NULL, *isow = NULL;
    CHECK(fp_op_tv_iso(2, NULL, &iso) == FP_OK);
    CHECK(fp_op_tv_aniso(2, NULL, &aniso) == FP_OK);
    double alpha[12];
    int64_t ashape[2] = {3, 4};
    for (int i = 0; i < 12; ++i) alpha[i] = 0.5 + 0.1 * i;
    fp_array al = {alpha, FP_F64, 2, ashape, NULL, FP_DEVICE_CPU};
    CHECK(fp_op_tv_iso_weighted(2, NULL, &al, &isow) == FP_OK);
    CHECK(fp_op_nparams(iso) == 2 && fp_op_nparams(isow) == 2 + 12);
    printf("names %s %s\n", fp_op_name(iso), fp_op_name(aniso));
    fp_op *bad = NULL;
    CHECK(fp_op_tv_iso(4, NULL, &bad) == FP_EPARAM);
    float x[2 * 3 * 4], z[2 * 3 * 4];
    for (int i = 0; i < 24; ++i) x[i] = (float)((i * 7) % 5) - 2.0f;
    int64_t shape[3] = {2, 3, 4};
    fp_array xa = {x, FP_F32, 3, shape, NULL, FP_DEVICE_CPU};
    fp_array za = {z, FP_F32, 3, shape, NULL, FP_DEVICE_CPU};
    fp_workspace *ws = NULL;
    fp_status s = fp_workspace_create(isow, &xa, &opt, &ws);
    if (!gpu) {
        CHECK(s == FP_EDEVICE || s == FP_OK);
        if (s == FP_OK) fp_workspace_free(ws);
        s = fp_prox(iso, 0.3, &xa, &za, &opt, NULL, NULL);
        CHECK(s == FP_EDEVICE);
        printf("no device: %s\n", fp_strerror(s));
    } else {
        CHECK(s == FP_OK);
        fp_info info;
        s = fp_prox(isow, 0.3, &xa, &za, &opt, ws, &info);
        CHECK(s == FP_OK || s == FP_ENOTCONV);
        double gaps[2], zerrs[2];
        int iters[2];
        CHECK(fp_workspace_image_info(ws, gaps, iters, zerrs, 2) == FP_OK);
        printf("solved: gap %g iters %d %d\n", info.gap, iters[0], iters[1]);
        fp_workspace_free(ws);
    }
    fp_op_free(iso);
    fp_op_free(aniso);
    fp_op_free(isow);
    printf("ok\n");
    return 0;
}
