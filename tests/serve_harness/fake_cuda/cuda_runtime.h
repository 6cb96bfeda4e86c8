// Minimal stand-in for the CUDA runtime API used by the serving loop's host
// code, so that luthe_b200/csrc/serve.cu can be compiled and exercised on a
// machine without a GPU (test infrastructure only).  Streams and events are
// synchronous: work "runs" when it is enqueued.
#pragma once
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorInvalidValue = 1, cudaErrorNotReady = 600, cudaErrorInvalidConfiguration = 9 };
typedef struct fake_stream *cudaStream_t;
typedef struct fake_event *cudaEvent_t;
typedef struct fake_graph *cudaGraph_t;
typedef struct fake_graph_exec *cudaGraphExec_t;
enum cudaMemcpyKind { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2, cudaMemcpyDeviceToDevice = 3 };
#define cudaStreamNonBlocking 1
#define cudaEventDisableTiming 2

static inline const char *cudaGetErrorString(cudaError_t) { return "fake"; }
static inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }
static inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
static inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind)
{
    memcpy(d, s, n);
    return cudaSuccess;
}
static inline cudaError_t cudaMemcpyAsync(void *d, const void *s, size_t n, cudaMemcpyKind, cudaStream_t)
{
    memcpy(d, s, n);
    return cudaSuccess;
}
static inline cudaError_t cudaMemset(void *d, int v, size_t n)
{
    memset(d, v, n);
    return cudaSuccess;
}
static inline cudaError_t cudaMallocHost(void **p, size_t n)
{
    *p = malloc(n);
    return *p ? cudaSuccess : 2;
}
static inline cudaError_t cudaFreeHost(void *p)
{
    free(p);
    return cudaSuccess;
}
static inline cudaError_t cudaStreamCreateWithFlags(cudaStream_t *s, unsigned)
{
    *s = (cudaStream_t)malloc(1);
    return cudaSuccess;
}
static inline cudaError_t cudaStreamDestroy(cudaStream_t s)
{
    free(s);
    return cudaSuccess;
}
static inline cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
static inline cudaError_t cudaStreamWaitEvent(cudaStream_t, cudaEvent_t, unsigned) { return cudaSuccess; }
// Events: an event recorded reports "not ready" for the next g_fake_event_lag
// queries (0 by default: work is complete as soon as it is enqueued), so that
// tests can keep PBS lanes busy across scheduler steps.
static int g_fake_event_lag = 0;
static inline cudaError_t cudaEventCreateWithFlags(cudaEvent_t *e, unsigned)
{
    *e = (cudaEvent_t)calloc(1, sizeof(int));
    return cudaSuccess;
}
static inline cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t)
{
    *(int *)e = g_fake_event_lag;
    return cudaSuccess;
}
static inline cudaError_t cudaEventQuery(cudaEvent_t e)
{
    int *left = (int *)e;
    if (*left > 0) {
        --*left;
        return cudaErrorNotReady;
    }
    return cudaSuccess;
}
static inline cudaError_t cudaEventDestroy(cudaEvent_t e)
{
    free(e);
    return cudaSuccess;
}
static inline cudaError_t cudaGraphExecDestroy(cudaGraphExec_t) { return cudaSuccess; }
