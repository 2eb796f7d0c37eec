/*
 * fftw3.h -- minimal FFTW3-compatible interface for building the reference
 * fftcorr C++ (cc/) without FFTW, which is not installed on this system.
 *
 * TEST INFRASTRUCTURE ONLY.  This header and shim_fft.c are part of the
 * oracle: they let the unmodified reference sources compile so that their
 * outputs can be used as the parity check and as the timed CPU baseline.
 * Nothing in the shipped fftcorr_b200 library links against it.
 *
 * Only the symbols the reference calls are declared:
 *   cc/grid/fft_grid.cc:81-84   fftw_plan_many_dft_r2c / _c2r (rank 3)
 *   cc/grid/fft_grid.cc:94-111  rank-2 r2c/c2r and rank-1 fftw_plan_many_dft
 *   cc/grid/fft_grid.cc:129,156 fftw_execute
 *   cc/grid/fft_grid.cc:137-171 fftw_execute_dft_r2c / _dft / _dft_c2r
 *   cc/grid/fft_grid.cc:54-66   fftw_destroy_plan, fftw_cleanup_threads
 *   cc/fftcorr.cc:325,453       wisdom import / export
 *   fftcorr/fftw/fftw.pyx:1-14  wisdom import / export / forget
 *
 * Conventions follow FFTW's documented ones: forward sign -1, backward +1,
 * transforms are unnormalised, r2c keeps n/2+1 outputs of the last dimension,
 * and c2r may overwrite its input.
 */
#ifndef FC_ORACLE_FFTW3_SHIM_H
#define FC_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fc_shim_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_CONSERVE_MEMORY (1U << 2)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_WISDOM_ONLY (1U << 21)

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride,
                                 int idist, fftw_complex *out,
                                 const int *onembed, int ostride, int odist,
                                 unsigned flags);

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed,
                                 int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist,
                                 unsigned flags);

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany,
                             fftw_complex *in, const int *inembed, int istride,
                             int idist, fftw_complex *out, const int *onembed,
                             int ostride, int odist, int sign, unsigned flags);

void fftw_execute(const fftw_plan p);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_destroy_plan(fftw_plan p);

void fftw_cleanup(void);
void fftw_cleanup_threads(void);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);

int fftw_import_wisdom_from_filename(const char *filename);
int fftw_export_wisdom_to_filename(const char *filename);
void fftw_forget_wisdom(void);

#ifdef __cplusplus
}
#endif

#endif /* FC_ORACLE_FFTW3_SHIM_H */
