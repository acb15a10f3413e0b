/* MoFFT serving loop (no counterpart in the reference): a request engine
 * that keeps plans, twiddles and staging buffers device-resident and runs
 * continuous batching on one GPU.
 *
 * Requests (length, batch, direction, FP32 or FP64, input, output) are
 * submitted from any thread and return a ticket at once.  A worker thread
 * admits pending requests while the device bytes they need (input + output
 * payload) fit in the HBM budget, coalesces every pending request of the same
 * (length, precision, direction) into ONE batched launch whose transforms
 * come from unrelated buffers (a device pointer table per launch), and runs
 * up to `streams` such launches concurrently, so requests that arrive while
 * others are on the GPU join the next launch as soon as a stream and memory
 * free up.  Buffers may be host memory (staged through pooled device memory;
 * pinned host memory overlaps best) or device memory (used in place).
 * Results are bit-identical whether a request runs alone or in a mix: every
 * transform of a given (length, precision, direction) runs the same kernel
 * and arithmetic regardless of what it is batched with. */
#ifndef MOFFT_SERVE_H
#define MOFFT_SERVE_H

#include "mofft.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mofft_server mofft_server;

typedef struct {
  size_t hbm_budget_bytes;      /* admission cap; 0 = 40 GiB */
  int streams;                  /* concurrent launches; 0 = 4 */
  size_t max_group_points;      /* points per coalesced launch; 0 = 2^27 */
} mofft_server_options;

typedef struct {
  size_t length;                /* 13-smooth, schedules of at most two passes */
  size_t batch;
  mofft_direction direction;
  int precision_bits;           /* 32 or 64 */
  const void *input;            /* batch * length complex values, dense */
  void *output;                 /* may equal input */
} mofft_request;

typedef struct {
  uint64_t submitted;
  uint64_t completed;
  uint64_t failed;
  uint64_t launches;            /* coalesced launches (each 1-2 kernels) */
  size_t peak_admitted_bytes;   /* largest admitted payload in flight */
} mofft_server_stats;

mofft_status mofft_server_create(mofft_server **server,
                                 const mofft_server_options *options);
/* Non-blocking; *ticket identifies the request.  The buffers must stay
 * valid until the request completes. */
mofft_status mofft_server_submit(mofft_server *server,
                                 const mofft_request *request,
                                 uint64_t *ticket);
/* Blocks until the request completes; returns its status and, if non-NULL,
 * the seconds from submission to completion on the GPU. */
mofft_status mofft_server_wait(mofft_server *server, uint64_t ticket,
                               double *latency_seconds);
/* Blocks until every submitted request has completed. */
mofft_status mofft_server_drain(mofft_server *server);
mofft_status mofft_server_get_stats(mofft_server *server,
                                    mofft_server_stats *stats);
void mofft_server_destroy(mofft_server *server);

#ifdef __cplusplus
}
#endif
#endif
