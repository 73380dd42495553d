// ecg_triples.h — closed-shell (T) and Lambda-(T) on the device.
#pragma once
#include "ecg_core.h"

namespace ecg {

// (T) / [T] for the amplitudes in c.T (calc_pertT_closed_shell,
// src/cc/cc_triples.jl:39-157).  With U1h/U2h (host, contravariant
// multipliers) the Lambda variant calc_ΛpertT_closed_shell (:159-295) is
// evaluated instead.
void pert_triples(Ctx& c, const double* U1h, const double* U2h, double* et, double* etb);

}  // namespace ecg
