// The library's internal interface between its flat solver entry points
// (gfix.cu) and GLU's own entry points (glu_abi.cu): how a solve's links
// reach the device and come back, and the phase marks of a call.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "../../include/glu_gfix.h"

namespace gfix {

// The links of one configuration -- V sites x 4 directions x 18 doubles in
// GLU's order -- moved between the caller's storage and the device buffer
// d_aos, ordered on stream s.  to_device may return before its copies are
// complete; to_host returns with the caller's storage written.  Both return
// 0, or -1 with the reason recorded for gfix_last_error().
class LinkIO {
 public:
  virtual int to_device(double *d_aos, size_t V, cudaStream_t s) = 0;
  virtual int to_host(const double *d_aos, size_t V, cudaStream_t s) = 0;

 protected:
  ~LinkIO() = default;
};

// gfix_landau, gfix_landau_driver, gfix_coulomb and gfix_coulomb_driver
// with the links moved by io
int landau_io(LinkIO &io, const size_t dims[4], const gfix_params *p,
              gfix_result *r);
int landau_driver_io(LinkIO &io, const size_t dims[4], const gfix_params *p,
                     gfix_result *r, double *obs, double *diag);
int coulomb_io(LinkIO &io, const size_t dims[4], const gfix_params *p,
               gfix_result *r, double *slice_theta, size_t *slice_iters);
int coulomb_driver_io(LinkIO &io, const size_t dims[4], const gfix_params *p,
                      gfix_result *r, double *obs_in, double *diag_in,
                      double *obs, double *diag);

// records "what: <CUDA error string>" for gfix_last_error(); returns -1
int cuda_failure(const char *what, cudaError_t e);

// GLU's restart and gauge-copy messages from the Landau solves of this
// thread (the flat entry points stay silent)
void set_restart_log(bool on);

// Phase marks of the *_io calls of this thread: fn(ctx, name) after each
// phase's work has completed on the device -- "engine" (workspaces ready),
// "to device", "solve", "post" (reunitarisation and diagnostics), "to
// host".  nullptr: no marks (and no synchronisation for them).
using PhaseMark = void (*)(void *ctx, const char *phase);
void set_phase_mark(PhaseMark fn, void *ctx);

}  // namespace gfix
