// family.cuh -- a parametric family of LPs solved together: every LP shares the constraint
// matrix, bounds and row senses; only the objective, its constant and the right-hand sides
// differ (the learned-warm-start configuration: one network, one A, many (b, c)).
//
// The single engine's iteration (solve_ipm, interior_point.cpp:454-740) runs in lockstep over a
// chunk of up to kFamilyWidth LPs whose vectors are interleaved, entry-major: v[i * W + k] is
// entry i of LP k. Every kernel maps threads to (entry, LP) with the LP index fastest, so a
// gather at a shared index (x[col[p]]) reads W consecutive doubles, and the shared structure --
// A, the normal matrix's sparse pattern, its minimum-degree (or nested-dissection) symbolic
// factor and the GPU work schedule -- is read once for all W LPs. The normal matrices A D_k A'
// share one pattern, so one symbolic analysis serves the whole family; the numeric L D L' runs
// level by level in one cooperative launch for the chunk, each level's work W times wider than a
// single LP's. Per-LP decisions (stopping test, best iterate, warm-start safeguard, iteration
// limits) are the single engine's, taken on the host from one read of the chunk's scalars per
// iteration. An LP that has finished leaves its slot, which the next LP of the family takes with
// its precomputed default start (or its kept supplied one), so the launch width stays full and a
// family's time follows its LPs' mean iteration count rather than each chunk's slowest LP.
#pragma once

#include "sov_ipm.h"

namespace sov {

constexpr int kFamilyWidth = 64;  // LPs per chunk

// Solves count LPs that share A, bounds and senses. Returns SOV_E_ARGUMENT when they do not.
int solve_family(int count, const sov_model* models, const sov_options* opt, int opt_stride, sov_result* results);

}  // namespace sov
