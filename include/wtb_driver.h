/*
 * wtb_driver.h -- deck-level entry of the BSE exciton + optics path (libwtbdriver.so).
 *
 * wtb_run() is the C++ counterpart of the reference program's BSE flow (wtb_main.f90:60-357
 * for BSE=T, BSE_BND=T, SPEC=T and PP_ONLY=T): it parses the stdin deck text with the
 * reference grammar (module_input_read.f90:235-663), reads PARAMS_FILE
 * (module_input_read.f90:32-176), runs the GPU stages through wtbgpu.h and writes the
 * reference's output files into OUTPUT / CALC_DATA.  The executable wtb_bse is
 * `wtb_bse < deck`, like `wtb.x < deck`.
 */
#ifndef WTB_DRIVER_H
#define WTB_DRIVER_H

#ifdef __cplusplus
extern "C" {
#endif

/* wall-clock seconds per stage of the last run (host view, including host<->device copies) */
typedef struct Timings {
  double bands;      /* model upload + k-mesh + bands */
  double sp;         /* velocity + single-particle table + sp_optics files */
  double build;      /* BSE kernel build */
  double solve;      /* dense solve + oscillators */
  double write_opt;  /* exciton wave-function files + bse_opt_diel files */
  double spectrum;   /* bse_opt_diel read-back + eps(omega) + bse_diel files */
  double total;      /* deck read to the last output file */
} Timings;

/* Run one deck.  Returns 0 on success; on failure 1, with the reference-style STOP message
 * in errbuf.  device selects the CUDA device; tm may be NULL. */
int wtb_run(const char* deck_text, int device, Timings* tm, char* errbuf, int errlen);

#ifdef __cplusplus
}
#endif
#endif
