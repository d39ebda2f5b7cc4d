// Entry points of the XPBD substep adjoint (pdem_xadj.cu) for the C ABI (pdem_xa_* in pdem_capi.cu).
// The adjoint runs on the plain FP64 path; the templates refuse every other instantiation.
#pragma once
#include <stdexcept>

#include "pdem_sim.cuh"

namespace pdem {

// start a recorded rollout from the state rows x (n x 3), q (n x 4), v, w (n x 3), device doubles
void xadjBegin(Sim<double>& S, const double* x, const double* q, const double* v, const double* w, int n);
// run `substeps` substeps of the production step, recording each one's start state, warm-start
// ledger and frozen active set
void xadjStep(Sim<double>& S, double dt, int substeps);
// current state rows (device doubles)
void xadjState(Sim<double>& S, double* x, double* q, double* v, double* w);
// gradients of L with respect to the recorded rollout's start state and (eN, eT, mu), given the
// adjoint of its end state (device doubles; theta on the host)
void xadjBackward(Sim<double>& S, const double* gx, const double* gq, const double* gv, const double* gw,
                  double* dx, double* dq, double* dv, double* dw, double* dtheta);
// [0] substeps recorded, [1] bytes held by the record, [2] bytes of the reverse workspace,
// [3] largest sweep count; err[0] the replay's largest position deviation from the recorded next
// state (in units of the global scale) over the last backward, err[1] the same for velocities (m/s)
void xadjInfo(Sim<double>& S, long* out, double* err);

// the record's discrete decisions, 7 per substep: contacts, manifolds, colours of the two
// colourings, main / stabilization / position sweeps; returns the number of substeps
long xadjSignature(Sim<double>& S, long* out, long cap);

// the branch signature of the record: a hash of every sweep update's branch decisions (impulse
// clamps, restitution cut-off, friction cone, active position contacts) over a replay
unsigned long long xadjBranches(Sim<double>& S);
template <class SIM>
unsigned long long xadjBranches(SIM&) {
  throw std::invalid_argument("the XPBD adjoint runs on the FP64 plain path (precision fp64)");
}
template <class SIM>
long xadjSignature(SIM&, long*, long) {
  throw std::invalid_argument("the XPBD adjoint runs on the FP64 plain path (precision fp64)");
}
template <class SIM>
void xadjBegin(SIM&, const double*, const double*, const double*, const double*, int) {
  throw std::invalid_argument("the XPBD adjoint runs on the FP64 plain path (precision fp64)");
}
template <class SIM>
void xadjStep(SIM&, double, int) {
  throw std::invalid_argument("the XPBD adjoint runs on the FP64 plain path (precision fp64)");
}
template <class SIM>
void xadjState(SIM&, double*, double*, double*, double*) {
  throw std::invalid_argument("the XPBD adjoint runs on the FP64 plain path (precision fp64)");
}
template <class SIM>
void xadjBackward(SIM&, const double*, const double*, const double*, const double*, double*, double*, double*,
                  double*, double*) {
  throw std::invalid_argument("the XPBD adjoint runs on the FP64 plain path (precision fp64)");
}
template <class SIM>
void xadjInfo(SIM&, long*, double*) {
  throw std::invalid_argument("the XPBD adjoint runs on the FP64 plain path (precision fp64)");
}

}  // namespace pdem
