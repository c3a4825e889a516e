/* Test infrastructure: C restatement of the reference SPB6_PC_IMEX stage loop.
 * Used only by tests/, smoke() and bench.py's CPU-baseline leg as the checker.
 *
 * int spb6_oracle_run(const spb6_case* c, const double* U0, void* out, size_t cap)
 *   runs the case (modes of spb6_case.h) and writes a result record followed by
 *   the arrays described in spb6_case.h into `out`.  Returns the number of
 *   bytes written, or a negative value if the case is rejected / cap too small.
 */
#ifndef SPB6_ORACLE_H
#define SPB6_ORACLE_H
#include <stddef.h>
#include "spb6_case.h"

#ifdef __cplusplus
extern "C" {
#endif
int spb6_oracle_run(const spb6_case* c, const double* U0, void* out, size_t cap);
#ifdef __cplusplus
}
#endif
#endif
