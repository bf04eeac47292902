/*
 * The discrete adjoint of the device layer (acDeviceLoadAdjoint,
 * acDeviceIntegrateSubstepAdjoint, the checkpoint-segment tape and the
 * parameter adjoints); its kernels are in adjoint.cu.
 */
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "internal.h"
#include "device_impl.h"

/* ---- discrete adjoint ---- */

/* The adjoint works in FP64 on the host layout (row pitch mx) for both
 * precisions: on an FP32-compensated device the forward states it linearises
 * about are the (hi, lo) pairs joined to doubles, and the reverse sweep, its
 * inner products and the parameter adjoints are FP64. */
static Geom
adj_geom(const Device d)
{
    return ac_make_geom(d->config, 0);
}

/* The 8 in-buffers of an FP32-compensated device joined to doubles in the
 * host layout, field q at q * cells of dst. */
static cudaError_t
join_state(const Device d, cudaStream_t st, double* dst, unsigned long long* launches)
{
    const Geom g64 = adj_geom(d);
    for (int q = 0; q < AC_NF; ++q) {
        const int b          = d->in_idx[q];
        const cudaError_t e  = ac_launch_join(d->geom, arr_hi(d, b, q), arr_lo(d, b, q),
                                              dst + (size_t)q * g64.cells, st, launches);
        if (e != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

static AcResult
ensure_adjoint(const Device d)
{
    if (d->config.int_params[AC_upwind]) {
        /* |u| in the upwinding terms has no derivative at u = 0; the reverse
         * pass covers the equations without them */
        fprintf(stderr, "astaroth_b200: the adjoint does not cover AC_upwind\n");
        return AC_FAILURE;
    }
    if (d->adj_lf)
        return AC_SUCCESS;
    const size_t fb = (size_t)adj_geom(d).cells * sizeof(double);
    AC_CUDA_CHECK(cudaMalloc((void**)&d->adj_lf, AC_NF * fb));
    AC_CUDA_CHECK(cudaMalloc((void**)&d->adj_lw, AC_NF * fb));
    AC_CUDA_CHECK(cudaMalloc((void**)&d->adj_mu, AC_MU_COUNT * fb));
    AC_CUDA_CHECK(cudaMalloc((void**)&d->adj_pgrad, 2 * sizeof(double)));
    AC_CUDA_CHECK(cudaMemset(d->adj_mu, 0, AC_MU_COUNT * fb));
    if (d->precision != 0) /* the joined in-buffers of a per-substep adjoint call */
        AC_CUDA_CHECK(cudaMalloc((void**)&d->adj_state, AC_NF * fb));
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceLoadAdjoint(const Device d, const Stream stream, const AcReal* const* lam_f)
{
    if (!d || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    if (ensure_adjoint(d) != AC_SUCCESS)
        return AC_FAILURE;
    cudaStream_t st   = d->streams[stream];
    const size_t cells = (size_t)adj_geom(d).cells;
    const size_t fb   = cells * sizeof(double);
    for (int q = 0; q < AC_NF; ++q) {
        if (lam_f && lam_f[q])
            AC_CUDA_CHECK(cudaMemcpyAsync(d->adj_lf + (size_t)q * cells, lam_f[q], fb,
                                          cudaMemcpyDeviceToDevice, st));
        else
            AC_CUDA_CHECK(cudaMemsetAsync(d->adj_lf + (size_t)q * cells, 0, fb, st));
    }
    AC_CUDA_CHECK(cudaMemsetAsync(d->adj_lw, 0, AC_NF * fb, st));
    AC_CUDA_CHECK(cudaMemsetAsync(d->adj_pgrad, 0, 2 * sizeof(double), st));
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceStoreAdjoint(const Device d, const Stream stream, AcReal* const* lam_f)
{
    if (!d || !lam_f || !stream_ok(stream) || !d->adj_lf)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const size_t cells = (size_t)adj_geom(d).cells;
    const size_t fb    = cells * sizeof(double);
    for (int q = 0; q < AC_NF; ++q)
        if (lam_f[q])
            AC_CUDA_CHECK(cudaMemcpyAsync(lam_f[q], d->adj_lf + (size_t)q * cells, fb,
                                          cudaMemcpyDeviceToDevice, d->streams[stream]));
    return AC_SUCCESS;
}

/* One adjoint substep about the state `state` (8 fields at q * cells, halos
 * filled), or about the in-buffers when state is NULL. */
static cudaError_t
launch_adjoint(const Device d, cudaStream_t st, const int step, const double dt,
               const double* state)
{
    StencilCoef sc;
    PhysConst pc;
    ac_make_stencil(d->config, &sc);
    ac_make_phys(d->config, &pc);
    const Geom g = adj_geom(d);
    if (!state && d->precision != 0) {
        const cudaError_t e = join_state(d, st, d->adj_state, &d->launches);
        if (e != cudaSuccess)
            return e;
        state = d->adj_state;
    }
    AdjointFields a;
    for (int q = 0; q < AC_NF; ++q) {
        a.f[q]  = state ? state + (size_t)q * g.cells : arr64(d, d->in_idx[q], q);
        a.lf[q] = d->adj_lf + (size_t)q * g.cells;
        a.lw[q] = d->adj_lw + (size_t)q * g.cells;
    }
    for (int m = 0; m < AC_MU_COUNT; ++m)
        a.mu[m] = d->adj_mu + (size_t)m * g.cells;
    const double alpha[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
    const double beta[3]  = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
    return ac_launch_adjoint_substep(g, a, sc, pc, alpha[step], beta[step], dt, d->adj_pgrad,
                                     st, &d->launches);
}

extern "C" AcResult
acDeviceIntegrateSubstepAdjoint(const Device d, const Stream stream, const int step_number,
                                const Volume start, const Volume end, const AcReal dt)
{
    if (!d || !stream_ok(stream) || step_number < 0 || step_number > 2 || !d->adj_lf)
        return AC_FAILURE;
    if (ensure_adjoint(d) != AC_SUCCESS)
        return AC_FAILURE;
    if (!is_whole_interior(d, start, end)) {
        fprintf(stderr, "astaroth_b200: acDeviceIntegrateSubstepAdjoint needs the whole interior\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    AC_CUDA_CHECK(launch_adjoint(d, d->streams[stream], step_number, dt, NULL));
    return AC_SUCCESS;
}

/* The launches of a tape recompute: per substep, halo fill, copy of the
 * in-block to the tape, substep, swap. */
static cudaError_t
record_tape(Device d, cudaStream_t st, const int steps, const double dt)
{
    const size_t state_elems = (size_t)AC_NF * adj_geom(d).cells;
    const Volume m0          = {0, 0, 0};
    const Volume m1          = {(size_t)d->geom.mx, (size_t)d->geom.my, (size_t)d->geom.mz};
    for (int n = 0; n < steps; ++n)
        for (int s = 0; s < 3; ++s) {
            cudaError_t e = launch_periodic(d, st, 0, AC_NF, m0, m1, NULL);
            if (e != cudaSuccess)
                return e;
            double* slot = d->adj_tape + (size_t)(3 * n + s) * state_elems;
            /* FP64: the 8 in-buffers are one contiguous block, one copy per state;
             * FP32 compensated: (hi, lo) joined to doubles */
            e = d->precision == 0
                    ? ac_launch_copy(arr64(d, d->in_idx[0], 0), slot, (long long)state_elems, st,
                                     NULL)
                    : join_state(d, st, slot, NULL);
            if (e != cudaSuccess)
                return e;
            e = launch_substep(d, st, s, dt, NULL);
            if (e != cudaSuccess)
                return e;
            acDeviceSwapBuffers(d);
        }
    return cudaSuccess;
}

extern "C" AcResult
acDeviceAdjointTapeForward(const Device d, const Stream stream, const int steps, const AcReal dt)
{
    if (!d || !stream_ok(stream) || steps < 1)
        return AC_FAILURE;
    const int blk = in_block_index(d);
    if (blk < 0) {
        fprintf(stderr, "astaroth_b200: the tape needs every field's in-buffer in one block\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    if (ensure_adjoint(d) != AC_SUCCESS)
        return AC_FAILURE;
    const size_t state_elems = (size_t)AC_NF * adj_geom(d).cells;
    if (d->adj_tape_states < 3 * steps) {
        AC_CUDA_CHECK(cudaDeviceSynchronize());
        invalidate_tape_graph(d);
        cudaFree(d->adj_tape);
        d->adj_tape        = NULL;
        d->adj_tape_states = 0;
        AC_CUDA_CHECK(cudaMalloc((void**)&d->adj_tape, 3 * (size_t)steps * state_elems *
                                                           sizeof(double)));
        d->adj_tape_states = 3 * steps;
    }
    cudaStream_t st = d->streams[stream];
    /* the recompute is one CUDA graph per in-block, kept for the next call
     * with the same steps, dt and stream (one capture per checkpoint length) */
    if (!(d->tape_valid[blk] && d->tape_steps[blk] == steps && d->tape_dt[blk] == dt &&
          d->tape_stream[blk] == (int)stream)) {
        if (d->tape_valid[blk])
            cudaGraphExecDestroy(d->tape_exec[blk]);
        d->tape_valid[blk] = 0;
        cudaGraph_t graph;
        AC_CUDA_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const cudaError_t rec = record_tape(d, st, steps, dt);
        const cudaError_t end = cudaStreamEndCapture(st, &graph);
        for (int q = 0; q < AC_NF; ++q) /* undo the capture's swaps */
            d->in_idx[q] = blk;
        AC_CUDA_CHECK(rec);
        AC_CUDA_CHECK(end);
        const cudaError_t inst = cudaGraphInstantiate(&d->tape_exec[blk], graph, 0);
        cudaGraphDestroy(graph);
        AC_CUDA_CHECK(inst);
        d->tape_valid[blk]  = 1;
        d->tape_steps[blk]  = steps;
        d->tape_dt[blk]     = dt;
        d->tape_stream[blk] = (int)stream;
    }
    AC_CUDA_CHECK(cudaGraphLaunch(d->tape_exec[blk], st));
    d->launches += (d->precision == 0 ? 9ull : 33ull) * steps; /* FP32: 8 joins per state */
    d->out_set = 0;
    if ((3 * steps) & 1) /* three swaps per step */
        acDeviceSwapBuffers(d);
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceAdjointTapeBackward(const Device d, const Stream stream, const int steps,
                            const AcReal dt)
{
    if (!d || !stream_ok(stream) || steps < 1)
        return AC_FAILURE;
    if (!d->adj_lf || d->adj_tape_states < 3 * steps) {
        fprintf(stderr,
                "astaroth_b200: acDeviceAdjointTapeBackward(%d steps) needs acDeviceLoadAdjoint "
                "and a tape of %d states (has %d)\n",
                steps, 3 * steps, d->adj_tape_states);
        return AC_FAILURE;
    }
    if (ensure_adjoint(d) != AC_SUCCESS)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    cudaStream_t st             = d->streams[stream];
    const size_t state_elems    = (size_t)AC_NF * adj_geom(d).cells;
    for (int n = steps - 1; n >= 0; --n)
        for (int s = 2; s >= 0; --s)
            AC_CUDA_CHECK(launch_adjoint(d, st, s, dt,
                                         d->adj_tape + (size_t)(3 * n + s) * state_elems));
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceGetParamAdjoints(const Device d, AcReal* nu_bar, AcReal* eta_bar)
{
    if (!d || !nu_bar || !eta_bar || !d->adj_pgrad)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    for (int s = 0; s < NUM_STREAMS; ++s)
        AC_CUDA_CHECK(cudaStreamSynchronize(d->streams[s]));
    double v[2];
    AC_CUDA_CHECK(cudaMemcpy(v, d->adj_pgrad, sizeof(v), cudaMemcpyDeviceToHost));
    *nu_bar  = v[0];
    *eta_bar = v[1];
    return AC_SUCCESS;
}

