/* Declarations of the MPFR 4.x entry points used to fit the EvalMod Chebyshev series in
 * 256-bit arithmetic (wg_evalmod_fit.cpp, and the reference's src/math/poly_approx.cpp when the
 * oracle recipe compiles it).
 *
 * The image carries the MPFR runtime (libmpfr.so.6) but not its development header, so this
 * header declares the public interface only: the documented mpfr_t record (precision, sign,
 * exponent, limb pointer) of LP64 builds, the rounding-mode enumeration, and one prototype per
 * function used; every function named here is an exported symbol of libmpfr.so.6, which the
 * builds link by its versioned name. */
#ifndef WG_ORACLE_MPFR_DECL_H
#define WG_ORACLE_MPFR_DECL_H

#ifdef __cplusplus
extern "C" {
#endif

typedef long mpfr_prec_t;
typedef int mpfr_sign_t;
typedef long mpfr_exp_t;
typedef unsigned long mp_limb_t;

typedef struct {
    mpfr_prec_t _mpfr_prec;
    mpfr_sign_t _mpfr_sign;
    mpfr_exp_t _mpfr_exp;
    mp_limb_t* _mpfr_d;
} __mpfr_struct;

typedef __mpfr_struct mpfr_t[1];
typedef __mpfr_struct* mpfr_ptr;
typedef const __mpfr_struct* mpfr_srcptr;

typedef enum {
    MPFR_RNDN = 0,
    MPFR_RNDZ,
    MPFR_RNDU,
    MPFR_RNDD,
    MPFR_RNDA,
    MPFR_RNDF,
    MPFR_RNDNA = -1
} mpfr_rnd_t;

void mpfr_init2(mpfr_ptr x, mpfr_prec_t prec);
void mpfr_clear(mpfr_ptr x);
void mpfr_swap(mpfr_ptr x, mpfr_ptr y);

int mpfr_set(mpfr_ptr rop, mpfr_srcptr op, mpfr_rnd_t rnd);
int mpfr_set_d(mpfr_ptr rop, double op, mpfr_rnd_t rnd);
int mpfr_set_si(mpfr_ptr rop, long op, mpfr_rnd_t rnd);
int mpfr_set_ui(mpfr_ptr rop, unsigned long op, mpfr_rnd_t rnd);
int mpfr_set_ui_2exp(mpfr_ptr rop, unsigned long op, mpfr_exp_t e, mpfr_rnd_t rnd);
int mpfr_set_str(mpfr_ptr rop, const char* s, int base, mpfr_rnd_t rnd);
double mpfr_get_d(mpfr_srcptr op, mpfr_rnd_t rnd);

int mpfr_add(mpfr_ptr rop, mpfr_srcptr a, mpfr_srcptr b, mpfr_rnd_t rnd);
int mpfr_sub(mpfr_ptr rop, mpfr_srcptr a, mpfr_srcptr b, mpfr_rnd_t rnd);
int mpfr_mul(mpfr_ptr rop, mpfr_srcptr a, mpfr_srcptr b, mpfr_rnd_t rnd);
int mpfr_div(mpfr_ptr rop, mpfr_srcptr a, mpfr_srcptr b, mpfr_rnd_t rnd);
int mpfr_neg(mpfr_ptr rop, mpfr_srcptr op, mpfr_rnd_t rnd);
int mpfr_abs(mpfr_ptr rop, mpfr_srcptr op, mpfr_rnd_t rnd);
int mpfr_cmp(mpfr_srcptr a, mpfr_srcptr b);
int mpfr_cos(mpfr_ptr rop, mpfr_srcptr op, mpfr_rnd_t rnd);
int mpfr_const_pi(mpfr_ptr rop, mpfr_rnd_t rnd);

#ifdef __cplusplus
}
#endif

#endif
