/*
 * Link-time companions of ref_shim.h for the compiled reference oracle
 * (test infrastructure only).
 *
 *  - check()/error(): same names and signatures as src/util/debug.cpp:5-16,
 *    but a failed check throws std::runtime_error instead of exit(0), so that a
 *    test sees the failure.
 *  - fft(), fftw_malloc(), fftw_free(): referenced only by corWavelet2D
 *    (src/util/wavelet.cpp:33-61), which no FD path calls.  FFTW is not
 *    installed here; these stubs abort if ever reached.
 */
#include "ref_shim.h"
#include <cstdlib>
#include <stdexcept>
#include "fftw3.h"

void check(bool eval, char *str)
{
  if (!eval)
    throw std::runtime_error(std::string("reference check failed: ") + (str ? str : ""));
}

void error(std::string errinfo)
{
  std::fprintf(stderr, "%s", errinfo.c_str());
}

void fft(int, int, fftw_complex *)
{
  std::fprintf(stderr, "fft stub reached: FFTW is not part of the FD path\n");
  std::abort();
}

extern "C" void *fftw_malloc(size_t)
{
  std::fprintf(stderr, "fftw_malloc stub reached: FFTW is not part of the FD path\n");
  std::abort();
}

extern "C" void fftw_free(void *)
{
  std::fprintf(stderr, "fftw_free stub reached: FFTW is not part of the FD path\n");
  std::abort();
}
