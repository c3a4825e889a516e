/* Test infrastructure: the reference harness's round-off probe.  Linked into
 * _ref/spb6_ref_ulp only, it interposes log, exp and pow: each returns the C
 * library's result moved one ulp up (nextafter towards +inf), or down when the
 * environment sets SPB6_ULP_DOWN.  A run of that
 * binary against the plain one measures how far the reference's own answer moves
 * under a one-ulp change in its libm calls -- the noise floor that a device
 * build, whose log / exp / pow round differently, is compared against. */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <math.h>

typedef double (*fn1)(double);
typedef double (*fn2)(double, double);

#include <pthread.h>
#include <stdlib.h>

static fn1 real_log, real_exp;
static fn2 real_pow;
static double towards = INFINITY;
static pthread_once_t once = PTHREAD_ONCE_INIT;

static void lookup(void) {  /* once, whichever OpenMP thread calls first */
    real_log = (fn1)dlsym(RTLD_NEXT, "log");
    real_exp = (fn1)dlsym(RTLD_NEXT, "exp");
    real_pow = (fn2)dlsym(RTLD_NEXT, "pow");
    towards = getenv("SPB6_ULP_DOWN") ? -INFINITY : INFINITY;
}
static void resolve(void) { pthread_once(&once, lookup); }

double log(double x) {
    resolve();
    return nextafter(real_log(x), towards);
}
double exp(double x) {
    resolve();
    return nextafter(real_exp(x), towards);
}
double pow(double x, double y) {
    resolve();
    return nextafter(real_pow(x, y), towards);
}
