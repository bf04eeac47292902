/*
 * A C caller of the device layer, in the shape of the reference's
 * samples/devicetest/main.cc:67-205: only the C header, the shared library
 * and libc.  It checks on one GPU
 *   1. the periodic boundary fill: every ghost cell equals its periodic image
 *      in the interior, bit for bit;
 *   2. that three RK3 steps as a loop of acDevicePeriodicBoundconds +
 *      acDeviceIntegrateSubstep + acDeviceSwapBuffers give the same bits as
 *      acDeviceIntegrateStep;
 *   3. reductions (max, min, sum) against the same reductions done here;
 *   4. the reference's argument checks (a sub-box substep is refused).
 * Prints "ac_devicetest: OK" and exits 0 when all hold.
 *
 *   ac_devicetest [nx ny nz]      (default 40 36 28)
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "astaroth_b200.h"

static int failures = 0;

#define CHECK(cond, ...)                                                                      \
    do {                                                                                      \
        if (!(cond)) {                                                                        \
            fprintf(stderr, "ac_devicetest: FAIL: " __VA_ARGS__);                             \
            fprintf(stderr, "\n");                                                            \
            ++failures;                                                                       \
        }                                                                                     \
    } while (0)

static int
wrap(const int v, const int n)
{
    const int r = v % n;
    return r < 0 ? r + n : r;
}

static size_t
idx(const int i, const int j, const int k, const int mx, const int my)
{
    return (size_t)i + (size_t)mx * ((size_t)j + (size_t)my * (size_t)k);
}

int
main(int argc, char** argv)
{
    int n[3] = {40, 36, 28};
    if (argc == 4)
        for (int a = 0; a < 3; ++a)
            n[a] = atoi(argv[1 + a]);

    AcMeshInfo info;
    if (acHostMeshInfoDefault(n[0], n[1], n[2], &info) != AC_SUCCESS)
        return 2;
    info.real_params[AC_nu_visc] = 5e-3;
    info.real_params[AC_eta]     = 5e-3;
    if (acHostUpdateParams(&info) != AC_SUCCESS)
        return 2;
    const int mx = info.int3_params[AC_mlocal].x, my = info.int3_params[AC_mlocal].y,
              mz = info.int3_params[AC_mlocal].z;
    const size_t cells = (size_t)mx * my * mz;

    AcMesh mesh, a, b;
    if (acHostMeshCreate(info, &mesh) != AC_SUCCESS || acHostMeshCreate(info, &a) != AC_SUCCESS ||
        acHostMeshCreate(info, &b) != AC_SUCCESS)
        return 2;
    acHostMeshRandomizeSeeded(&mesh, 7, 1e-5, 1e-3, 1e-4);

    Device dev;
    if (acDeviceCreate(0, info, &dev) != AC_SUCCESS) {
        fprintf(stderr, "ac_devicetest: acDeviceCreate failed\n");
        return 2;
    }
    const Volume m0 = {0, 0, 0}, m1 = {(size_t)mx, (size_t)my, (size_t)mz};
    const Volume n0 = {NGHOST, NGHOST, NGHOST};
    const Volume n1 = {(size_t)(n[0] + NGHOST), (size_t)(n[1] + NGHOST), (size_t)(n[2] + NGHOST)};
    const AcReal dt = 1e-3;

    /* 1. periodic fill */
    CHECK(acDeviceLoadMesh(dev, STREAM_DEFAULT, mesh) == AC_SUCCESS, "load");
    CHECK(acDevicePeriodicBoundconds(dev, STREAM_DEFAULT, m0, m1) == AC_SUCCESS, "boundconds");
    CHECK(acDeviceStoreMesh(dev, STREAM_DEFAULT, &a) == AC_SUCCESS, "store");
    long bad = 0;
    for (int q = 0; q < NUM_VTXBUF_HANDLES; ++q)
        for (int k = 0; k < mz; ++k)
            for (int j = 0; j < my; ++j)
                for (int i = 0; i < mx; ++i) {
                    const int si = NGHOST + wrap(i - NGHOST, n[0]);
                    const int sj = NGHOST + wrap(j - NGHOST, n[1]);
                    const int sk = NGHOST + wrap(k - NGHOST, n[2]);
                    if (a.vertex_buffer[q][idx(i, j, k, mx, my)] !=
                        a.vertex_buffer[q][idx(si, sj, sk, mx, my)])
                        ++bad;
                }
    CHECK(bad == 0, "%ld ghost cells differ from their periodic images", bad);

    /* 2. substep loop against the graph-captured step */
    CHECK(acDeviceLoadMesh(dev, STREAM_DEFAULT, mesh) == AC_SUCCESS, "load");
    for (int step = 0; step < 3; ++step)
        for (int s = 0; s < 3; ++s) {
            acDevicePeriodicBoundconds(dev, STREAM_DEFAULT, m0, m1);
            CHECK(acDeviceIntegrateSubstep(dev, STREAM_DEFAULT, s, n0, n1, dt) == AC_SUCCESS,
                  "substep %d", s);
            acDeviceSwapBuffers(dev);
        }
    CHECK(acDeviceSynchronizeStream(dev, STREAM_ALL) == AC_SUCCESS, "synchronize");
    CHECK(acDeviceStoreMesh(dev, STREAM_DEFAULT, &a) == AC_SUCCESS, "store");
    CHECK(acDeviceLoadMesh(dev, STREAM_DEFAULT, mesh) == AC_SUCCESS, "load");
    for (int step = 0; step < 3; ++step)
        CHECK(acDeviceIntegrateStep(dev, STREAM_DEFAULT, dt) == AC_SUCCESS, "step");
    CHECK(acDeviceSynchronizeStream(dev, STREAM_ALL) == AC_SUCCESS, "synchronize");
    CHECK(acDeviceStoreMesh(dev, STREAM_DEFAULT, &b) == AC_SUCCESS, "store");
    bad = 0;
    for (int q = 0; q < NUM_VTXBUF_HANDLES; ++q)
        for (int k = NGHOST; k < n[2] + NGHOST; ++k)
            for (int j = NGHOST; j < n[1] + NGHOST; ++j)
                for (int i = NGHOST; i < n[0] + NGHOST; ++i) {
                    const size_t c = idx(i, j, k, mx, my);
                    if (memcmp(&a.vertex_buffer[q][c], &b.vertex_buffer[q][c], sizeof(AcReal)))
                        ++bad;
                }
    CHECK(bad == 0, "%ld interior values differ between the substep loop and the step", bad);
    bad = 0;
    for (int q = 0; q < NUM_VTXBUF_HANDLES; ++q)
        for (size_t c = 0; c < cells; ++c)
            if (!isfinite(b.vertex_buffer[q][c]))
                ++bad;
    CHECK(bad == 0, "%ld values are not finite", bad);

    /* 3. reductions of the interior of field uux against the same here */
    AcReal vmax = -INFINITY, vmin = INFINITY, vsum = 0;
    for (int k = NGHOST; k < n[2] + NGHOST; ++k)
        for (int j = NGHOST; j < n[1] + NGHOST; ++j)
            for (int i = NGHOST; i < n[0] + NGHOST; ++i) {
                const AcReal v = b.vertex_buffer[VTXBUF_UUX][idx(i, j, k, mx, my)];
                vmax           = v > vmax ? v : vmax;
                vmin           = v < vmin ? v : vmin;
                vsum += v;
            }
    AcReal r;
    CHECK(acDeviceReduceScal(dev, STREAM_DEFAULT, RTYPE_MAX, VTXBUF_UUX, &r) == AC_SUCCESS &&
              r == vmax,
          "RTYPE_MAX %.17g against %.17g", r, vmax);
    CHECK(acDeviceReduceScal(dev, STREAM_DEFAULT, RTYPE_MIN, VTXBUF_UUX, &r) == AC_SUCCESS &&
              r == vmin,
          "RTYPE_MIN %.17g against %.17g", r, vmin);
    CHECK(acDeviceReduceScal(dev, STREAM_DEFAULT, RTYPE_SUM, VTXBUF_UUX, &r) == AC_SUCCESS &&
              fabs(r - vsum) <= 1e-12 * (fabs(vmax) + fabs(vmin)) * (double)n[0] * n[1] * n[2],
          "RTYPE_SUM %.17g against %.17g", r, vsum);

    /* 4. argument checks */
    const Volume sub = {NGHOST + 1, NGHOST, NGHOST};
    CHECK(acDeviceIntegrateSubstep(dev, STREAM_DEFAULT, 0, sub, n1, dt) == AC_FAILURE,
          "a sub-box substep was accepted");
    CHECK(acDeviceIntegrateSubstep(dev, STREAM_DEFAULT, 3, n0, n1, dt) == AC_FAILURE,
          "substep 3 was accepted");

    CHECK(acDeviceDestroy(&dev) == AC_SUCCESS && dev == NULL, "destroy");
    acHostMeshDestroy(&mesh);
    acHostMeshDestroy(&a);
    acHostMeshDestroy(&b);
    if (failures) {
        fprintf(stderr, "ac_devicetest: %d check(s) failed\n", failures);
        return 1;
    }
    printf("ac_devicetest: OK (%d x %d x %d, %s)\n", n[0], n[1], n[2], acB200Version());
    return 0;
}
