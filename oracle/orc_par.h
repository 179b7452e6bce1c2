#ifndef ORC_PAR_H
#define ORC_PAR_H
#include <stdint.h>
typedef void (*orc_range_fn)(void *ctx, uint64_t begin, uint64_t end);
int orc_threads(void);
void orc_parallel(uint64_t n, uint64_t grain, orc_range_fn fn, void *ctx);
#endif
