/* A small pthreads parallel-for for the oracle's independent loops (rays, pixels, probes).  Chunks of `grain`
 * indices are handed out from an atomic counter; each index is computed exactly as the sequential loop would, so
 * the results do not depend on the thread count.  ORC_THREADS sets the thread count (default: online CPUs). */
#include <pthread.h>
#include <stdlib.h>
#include <unistd.h>
#include "orc_par.h"

typedef struct {
  uint64_t n, grain;
  uint64_t next;
  orc_range_fn fn;
  void *ctx;
} job_t;

static void *worker(void *arg) {
  job_t *j = (job_t *)arg;
  for (;;) {
    uint64_t b = __atomic_fetch_add(&j->next, j->grain, __ATOMIC_RELAXED);
    if (b >= j->n) break;
    uint64_t e = b + j->grain < j->n ? b + j->grain : j->n;
    j->fn(j->ctx, b, e);
  }
  return NULL;
}

int orc_threads(void) {
  const char *s = getenv("ORC_THREADS");
  if (s && atoi(s) > 0) return atoi(s);
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 1;
}

void orc_parallel(uint64_t n, uint64_t grain, orc_range_fn fn, void *ctx) {
  int nt = orc_threads();
  if (grain == 0) grain = 1;
  if (nt <= 1 || n <= grain) { if (n) fn(ctx, 0, n); return; }
  if (nt > 256) nt = 256;
  job_t j = {n, grain, 0, fn, ctx};
  pthread_t th[256];
  int started = 0;
  for (int i = 1; i < nt; i++)
    if (pthread_create(&th[started], NULL, worker, &j) == 0) started++;
  worker(&j);
  for (int i = 0; i < started; i++) pthread_join(th[i], NULL);
}
