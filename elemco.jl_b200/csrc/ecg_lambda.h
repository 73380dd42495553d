// ecg_lambda.h — closed-shell CCSD/DCSD Lambda (left-hand) equations on the device.
#pragma once
#include "ecg_core.h"

namespace ecg {

struct LambdaResult {
  double norm = 0, normR = 0, dnorm = 0;
  int iterations = 0;
  bool converged = false;
};

// Dress with the current T1 and build v_{mb}^{cd} T^{ij}_{cd}
// (lm_cc_iterations! setup, src/cc/cc_lagrange.jl:1163-1167, :948-952).
void lambda_prepare(Ctx& c, bool dc);
void lambda_load_U(Ctx& c, const double* U1h, const double* U2h);
void lambda_store_U(Ctx& c, double* U1h, double* U2h);
void lambda_store_R(Ctx& c, double* R1h, double* R2h);
// RU = calc_ccsd_vector_times_Jacobian(U) (cc_lagrange.jl:9-220), DF form.
void lambda_residual(Ctx& c, bool dc);
// lm_cc_iterations! (cc_lagrange.jl:1155-1223) starting from
// transform_amplitudes2lagrange_multipliers! (cctools.jl:887-930).
LambdaResult lambda_solve(Ctx& c, bool dc, const ecg_cc_opts& o);
// calc_1RDM (cc_lagrange.jl:793-848) for U in c.U; host outputs may be NULL.
void one_rdm(Ctx& c, double* D1h, double* dD1h);

}  // namespace ecg
