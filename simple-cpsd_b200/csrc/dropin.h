// dropin.h -- the drop-in cpsd()'s calls from capi.cu into engine.cu.
#pragma once

#include <cstddef>

struct cpsd_gpu_ctx;

// The tables of cpsd_gpu_set_tables as the reference passes them (grids on
// the half box, one set per kind).
struct TableArgs {
    const int *katm;
    const double *amass, *zv, *rcell, *G, *tg, *vc, *vg;
    const int *lmmax;
    const double *vnlnrm, *vl, *vnl;
};

// What a call that reuses the context verifies on host threads while its
// steps run: the caller's mask against the context's, the caller's tables
// against the ones on the device.  A mismatch discards the steps' results
// (nothing is written to the caller) and returns kDropinRedo.
struct DropinCheck {
    const int *masker;      // the caller's (2 nfft3d values)
    const int *masker_ref;  // the context's
    size_t masker_n;
    TableArgs tables;
};
constexpr int kDropinRedo = -1;

// c2's sphere gathered and uploaded, the steps started at once, c2's zeros
// outside the sphere (and the DropinCheck, when given) checked beside them,
// then the outputs in the reference's layout.
int cpsd_dropin_state_run_fetch(cpsd_gpu_ctx *c, const double *r2in, int inner, int move, double *E,
                                double *deltae, double *deltac, double *deltar, double *c1, double *c2,
                                double *cpsi, double *dn, double *hml, double *lmd, double *r1, double *r2,
                                double *fion, const DropinCheck *check);

// cpsd_gpu_run, then the host-layout outputs, with c1 and cpsi zeroed on
// host threads during the run (c2 must have just gone through
// cpsd_gpu_set_state).
int cpsd_dropin_run_fetch(cpsd_gpu_ctx *c, int inner, int move, double *E, double *deltae, double *deltac,
                          double *deltar, double *c1, double *c2, double *cpsi, double *dn, double *hml,
                          double *lmd, double *r1, double *r2, double *fion);
