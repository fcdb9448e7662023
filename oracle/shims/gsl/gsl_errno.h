/*
 * Stand-in for the GSL error-handler switch the reference calls
 * (curved_boundaries.C:113).  Oracle build only.
 */
#ifndef ORACLE_SHIM_GSL_ERRNO_H
#define ORACLE_SHIM_GSL_ERRNO_H
#ifdef __cplusplus
extern "C" {
#endif
typedef void gsl_error_handler_t(const char *reason, const char *file,
                                 int line, int gsl_errno);
gsl_error_handler_t *gsl_set_error_handler_off(void);
#ifdef __cplusplus
}
#endif
#endif
