/* A plain C caller of the library, linked the way a cgo, JNI or N-API
 * binding links it: compiled as C99 against include/ct2b200.h, linked to
 * libct2b200.so.  It calls only what needs no GPU -- argument checks that
 * come before any CUDA call, empty inputs, host-side bookkeeping -- so it
 * runs on a machine without one.  Exit status 0 when every check holds. */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "ct2b200.h"

static int fails = 0;

#define CHECK(cond)                                                            \
    do {                                                                       \
        if (!(cond)) {                                                         \
            fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
            fails++;                                                           \
        }                                                                      \
    } while (0)

int main(void)
{
    CHECK(strstr(ct2_version(), "sm_100a") != NULL);

    /* a bad argument: the status code and the thread's message */
    CHECK(ct2_set_backprojector(2) == CT2_EINVAL);
    CHECK(strlen(ct2_last_error()) > 0);
    CHECK(ct2_set_backprojector(0) == CT2_OK);

    /* host bookkeeping */
    unsigned long long launches = 1;
    CHECK(ct2_launch_count(&launches, 1) == CT2_OK);
    CHECK(ct2_launch_count(&launches, 0) == CT2_OK && launches == 0);
    CHECK(ct2_launch_count(NULL, 0) == CT2_EINVAL);

    /* the projector's host entry point: shape errors before any device work,
     * an empty sinogram is no work */
    float fv[2 * 18] = {0};
    float vol[27] = {0};
    float sino[2 * 4 * 4];
    CHECK(ct2_view_proj3D_sinoproj_linear(sino, NULL, fv, 2, 4, 4, 1.f, 1.f, -2.f, -2.f, vol, 1.f,
                                          1.f, 1.f, 0.f, 0.f, 0.f, -3, 3, 3) == CT2_EINVAL);
    CHECK(strstr(ct2_last_error(), "dimensions") != NULL);
    CHECK(ct2_view_proj3D_sinoproj_linear(sino, NULL, fv, 2, 4, 4, 1.f, 0.f, -2.f, -2.f, vol, 1.f,
                                          1.f, 0.f, 0.f, 0.f, 0.f, 3, 3, 3) == CT2_EINVAL);
    CHECK(ct2_view_proj3D_sinoproj_linear(sino, NULL, fv, 0, 4, 4, 1.f, 1.f, -2.f, -2.f, vol, 1.f,
                                          1.f, 1.f, 0.f, 0.f, 0.f, 3, 3, 3) == CT2_OK);

    /* the multi-volume device entry points */
    CHECK(ct2_dev_view_proj3D_sinoproj_linear_many(-1, NULL, NULL, 2, 4, 4, 1.f, 1.f, -2.f, -2.f,
                                                   NULL, 1.f, 1.f, 1.f, 0.f, 0.f, 0.f, 3, 3, 3,
                                                   NULL) == CT2_EINVAL);
    CHECK(ct2_dev_view_proj3D_sinobackproject_linear_many(0, NULL, NULL, 2, 4, 4, 1.f, 1.f, -2.f,
                                                          -2.f, NULL, 1.f, 1.f, 1.f, 0.f, 0.f, 0.f,
                                                          3, 3, 3, NULL) == CT2_OK);

    /* the batch engine's handle checks */
    void* handle = NULL;
    CHECK(ct2_batch_create(0, &handle) == CT2_EINVAL && handle == NULL);
    CHECK(ct2_batch_commit(NULL, NULL, NULL) == CT2_EINVAL);
    CHECK(ct2_batch_destroy(NULL) == CT2_OK);

    if (fails == 0) printf("c caller: all checks hold\n");
    return fails == 0 ? 0 : 1;
}
