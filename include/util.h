/* util.h — small numeric helpers and raw binary I/O.
 *
 * Same declarations as upstream include/util.h:37-84.  ReadData checks that
 * the file holds exactly n*size bytes (upstream src/util.c:33-63) and returns
 * -1 (open), -2 (size mismatch) or -3 (short read); WriteData writes or
 * appends n items (src/util.c:70-91).
 */
#ifndef UTIL_H
#define UTIL_H

#include <math.h>
#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

static inline double square(const double x) { return x*x; }

static inline double maxf(const double x, const double y) { return (x >= y) ? x : y; }

static inline double minf(const double x, const double y) { return (x <= y) ? x : y; }

int ReadData(const char *filename, void *data, const size_t size, const size_t n);

int WriteData(const char *filename, const void *data, const size_t size, const size_t n, const bool append);

#ifdef __cplusplus
}
#endif

#endif /* UTIL_H */
