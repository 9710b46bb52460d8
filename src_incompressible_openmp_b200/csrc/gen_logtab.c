/* Generates logtab.inc: log(j/128) for j = 88..184 as double-double (hi, lo),
 * plus ln2 split so that k*LN2_HI is exact for |k| < 2^11.
 * Computed in IEEE binary128 (gcc __float128 + libquadmath).
 * Build: gcc -O2 gen_logtab.c -lquadmath -o gen_logtab && ./gen_logtab > logtab.inc */
#include <stdio.h>
#include <quadmath.h>
static void split(__float128 v, double* hi, double* lo) {
    *hi = (double)v;
    *lo = (double)(v - (__float128)(*hi));
}
int main(void) {
    printf("/* generated by gen_logtab.c: log(j/128), j = 88..184, as (hi, lo) */\n");
    printf("#define MPCD_LOGTAB_J0 88\n#define MPCD_LOGTAB_N 97\n");
    printf("MPCD_LOGTAB_QUAL double mpcd_logtab[MPCD_LOGTAB_N][2] = {\n");
    for (int j = 88; j <= 184; ++j) {
        double hi, lo;
        split(logq((__float128)j / 128), &hi, &lo);
        printf("  {%a, %a},\n", hi, lo);
    }
    printf("};\n");
    __float128 ln2 = logq((__float128)2);
    /* ln2_hi keeps 42 significant bits so that k * ln2_hi is exact for |k| < 2^11 */
    double hi = (double)ln2;
    union { double d; unsigned long long u; } c; c.d = hi; c.u &= ~((1ULL << 11) - 1); hi = c.d;
    __float128 rem = ln2 - (__float128)hi;
    double lo = (double)rem;
    printf("#define MPCD_LN2_HI %a\n#define MPCD_LN2_LO %a\n", hi, lo);
    return 0;
}
