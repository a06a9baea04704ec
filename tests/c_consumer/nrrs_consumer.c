/*
 * A plain C consumer of the library's C-ABI (include/nrrs.h): the code a C host, or a cgo or
 * ctypes binding, compiles against the header. It runs one depth of the path:
 * - synthetic vertices on the host (nrrs_synth_vertices), copied to the device;
 * - nrrs_step (inference, normalisation, decision, emission);
 * - the queue size, the queue and the device status read back;
 * - nrrs_decide_emit on the step's own factors, which must emit the same queue bit for bit.
 *
 * Usage: nrrs_consumer [n]. Exit codes: 0 on success, 2 when no sm_100 device is present
 * (nothing runs), 1 on any failure.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "nrrs.h"

#define FAIL(...)                         \
    do {                                  \
        fprintf(stderr, __VA_ARGS__);     \
        fputc('\n', stderr);              \
        return 1;                         \
    } while (0)
#define CUDA(x)                                                                   \
    do {                                                                          \
        cudaError_t e_ = (x);                                                     \
        if (e_ != cudaSuccess) FAIL("%s: %s", #x, cudaGetErrorString(e_));        \
    } while (0)
#define NRRS(ctx, x)                                                                          \
    do {                                                                                      \
        int rc_ = (x);                                                                        \
        if (rc_ != NRRS_OK)                                                                   \
            FAIL("%s: %s (%s)", #x, nrrs_status_string(rc_), (ctx) ? nrrs_last_error(ctx) : ""); \
    } while (0)

static void* to_device(const void* host, size_t bytes, int* ok) {
    void* d = NULL;
    if (cudaMalloc(&d, bytes ? bytes : 4) != cudaSuccess) { *ok = 0; return NULL; }
    if (bytes && cudaMemcpy(d, host, bytes, cudaMemcpyHostToDevice) != cudaSuccess) *ok = 0;
    return d;
}

int main(int argc, char** argv) {
    const uint32_t n = argc > 1 ? (uint32_t)strtoul(argv[1], NULL, 10) : 100000u;
    if (n == 0) FAIL("n must be positive");
    if (nrrs_device_available() != 1) {
        printf("no sm_100 device: nothing run\n");
        return 2;
    }

    nrrs_config cfg;
    nrrs_config_default(&cfg);
    cfg.precision = NRRS_PREC_FP16;
    cfg.max_queue = n;
    cfg.max_train = 1u << 16;
    nrrs_ctx* ctx = NULL;
    NRRS(ctx, nrrs_create(&cfg, &ctx));
    NRRS(ctx, nrrs_set_step(ctx, 3));

    /* host vertices */
    float* pos = malloc(12 * (size_t)n);
    float* wi = malloc(12 * (size_t)n);
    float* nrm = malloc(12 * (size_t)n);
    float* rough = malloc(4 * (size_t)n);
    float* alb = malloc(12 * (size_t)n);
    float* thp = malloc(12 * (size_t)n);
    uint32_t* depth = malloc(4 * (size_t)n);
    float* rnd = malloc(4 * (size_t)n);
    if (!pos || !wi || !nrm || !rough || !alb || !thp || !depth || !rnd) FAIL("host allocation");
    nrrs_synth_vertices(7, 0, n, pos, wi, nrm, rough, alb, thp, depth, rnd, NULL, NULL);

    int ok = 1;
    nrrs_vertex_soa v;
    memset(&v, 0, sizeof(v));
    v.pos = to_device(pos, 12 * (size_t)n, &ok);
    v.wi = to_device(wi, 12 * (size_t)n, &ok);
    v.normal = to_device(nrm, 12 * (size_t)n, &ok);
    v.roughness = to_device(rough, 4 * (size_t)n, &ok);
    v.albedo = to_device(alb, 12 * (size_t)n, &ok);
    v.thp = to_device(thp, 12 * (size_t)n, &ok);
    v.depth = to_device(depth, 4 * (size_t)n, &ok);
    float* d_rnd = to_device(rnd, 4 * (size_t)n, &ok);
    if (!ok) FAIL("device copies");

    const uint32_t cap = 9u * n;
    float *stats = NULL, *rrs = NULL, *rrs_norm = NULL, *rrs_norm2 = NULL;
    uint8_t *split = NULL, *split2 = NULL;
    uint32_t *queue = NULL, *queue2 = NULL, *size_dev = NULL;
    CUDA(cudaMalloc((void**)&stats, 12 * (size_t)n));
    CUDA(cudaMalloc((void**)&rrs, 4 * (size_t)n));
    CUDA(cudaMalloc((void**)&rrs_norm, 4 * (size_t)n));
    CUDA(cudaMalloc((void**)&rrs_norm2, 4 * (size_t)n));
    CUDA(cudaMalloc((void**)&split, n));
    CUDA(cudaMalloc((void**)&split2, n));
    CUDA(cudaMalloc((void**)&queue, 4 * (size_t)cap));
    CUDA(cudaMalloc((void**)&queue2, 4 * (size_t)cap));
    CUDA(cudaMalloc((void**)&size_dev, 8));

    nrrs_decide_params dp;
    nrrs_decide_params_default(&dp);
    NRRS(ctx, nrrs_step(ctx, &v, d_rnd, n, n, 0, &dp, stats, rrs, rrs_norm, split, queue, cap,
                        size_dev, NULL));
    NRRS(ctx, nrrs_decide_emit(ctx, rrs, d_rnd, NULL, n, n, 0, NULL, &dp, rrs_norm2, split2,
                               queue2, cap, size_dev + 1, NULL));
    uint32_t flags = 0;
    NRRS(ctx, nrrs_get_device_status(ctx, &flags, NULL));
    if (flags) FAIL("device status flags 0x%x", flags);

    uint32_t sizes[2];
    CUDA(cudaMemcpy(sizes, size_dev, 8, cudaMemcpyDeviceToHost));
    if (sizes[0] == 0 || sizes[0] > cap) FAIL("queue size %u out of range", sizes[0]);
    if (sizes[1] != sizes[0]) FAIL("nrrs_decide_emit emitted %u, nrrs_step %u", sizes[1], sizes[0]);
    uint32_t* q1 = malloc(4 * (size_t)sizes[0]);
    uint32_t* q2 = malloc(4 * (size_t)sizes[0]);
    float* f1 = malloc(4 * (size_t)n);
    float* f2 = malloc(4 * (size_t)n);
    if (!q1 || !q2 || !f1 || !f2) FAIL("host allocation");
    CUDA(cudaMemcpy(q1, queue, 4 * (size_t)sizes[0], cudaMemcpyDeviceToHost));
    CUDA(cudaMemcpy(q2, queue2, 4 * (size_t)sizes[0], cudaMemcpyDeviceToHost));
    CUDA(cudaMemcpy(f1, rrs_norm, 4 * (size_t)n, cudaMemcpyDeviceToHost));
    CUDA(cudaMemcpy(f2, rrs_norm2, 4 * (size_t)n, cudaMemcpyDeviceToHost));
    if (memcmp(q1, q2, 4 * (size_t)sizes[0]) != 0) FAIL("emitted queues differ");
    if (memcmp(f1, f2, 4 * (size_t)n) != 0) FAIL("normalised factors differ");
    for (uint32_t j = 1; j < sizes[0]; ++j)
        if (q1[j] < q1[j - 1] || q1[j] >= n) FAIL("queue not in vertex order at %u", j);

    printf("ok n=%u emitted=%u launches=%llu\n", n, sizes[0],
           (unsigned long long)nrrs_launch_count(ctx));
    free(q1); free(q2); free(f1); free(f2);
    free(pos); free(wi); free(nrm); free(rough); free(alb); free(thp); free(depth); free(rnd);
    cudaFree((void*)v.pos); cudaFree((void*)v.wi); cudaFree((void*)v.normal);
    cudaFree((void*)v.roughness); cudaFree((void*)v.albedo); cudaFree((void*)v.thp);
    cudaFree((void*)v.depth); cudaFree(d_rnd); cudaFree(stats); cudaFree(rrs);
    cudaFree(rrs_norm); cudaFree(rrs_norm2); cudaFree(split); cudaFree(split2);
    cudaFree(queue); cudaFree(queue2); cudaFree(size_dev);
    nrrs_destroy(ctx);
    return 0;
}
