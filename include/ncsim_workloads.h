/*
 * ncsim_workloads.h — seeded synthetic workloads (libncsim_workloads.so).
 *
 * The circuits the benchmark and the tests run: not part of the drop-in
 * interface of ncsim_cuda.h, which a program that brings its own circuits
 * needs alone.  The library links against libncsim_cuda.so and returns that
 * library's handles (free them with ncsim_circuit_free / ncsim_batch_free).
 * Every choice is drawn from StdRng::seed_from_u64(seed) (rand 0.8) or from
 * the caller's generator, in the order of the CPU oracle's generators.
 */
#ifndef NCSIM_WORKLOADS_H
#define NCSIM_WORKLOADS_H

#include "ncsim_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Seeded synthetic workloads (StdRng::seed_from_u64(seed) draws every choice).
 * Random layer family: per layer one of {H, S, T, SQRT_X, RZ(theta)} on every
 * qubit, then CZ on a random perfect matching (optionally followed by
 * DEPOLARIZE2(noise_p)); Z measurements of qubits [m_lo, m_hi) at the end. */
ncsim_status ncsim_workload_random_circuit(uint32_t n, uint32_t depth, uint64_t seed, double noise_p, uint32_t m_lo,
                                           uint32_t m_hi, ncsim_circuit** out);
/* The same family drawn from the caller's generator, which keeps its state
 * (a noisy trajectory draws its circuit and then its noise and measurement
 * outcomes from one StdRng). */
ncsim_status ncsim_workload_random_circuit_rng(ncsim_rng* rng, uint32_t n, uint32_t depth, double noise_p,
                                               uint32_t m_lo, uint32_t m_hi, ncsim_circuit** out);
/* Permutation/diagonal family: H on min(16, n) qubits, then `gates` gates
 * from {CX, CCX, CCZ, DIAG over the register, MONOMIAL on 8 qubits}. */
ncsim_status ncsim_workload_reversible_circuit(uint32_t n, uint32_t gates, uint64_t seed, ncsim_circuit** out);

/* The frame-sampler benchmark circuit (ncsim's examples/bench.rs:264-294 with
 * n = 1000, rounds = 20, meas = 100, p = 1e-3, seed = 9): H on qubits 0..n/2;
 * per round CX(q, b) and DEPOLARIZE2(p) on (q, b) for every even q, with
 * b = (q + 1 + gen_range(0..n-1)) mod n, then `meas` Z measurements of
 * gen_range(0..n) qubits. */
ncsim_status ncsim_workload_frames_circuit(uint32_t n, uint32_t rounds, uint32_t meas, double p, uint64_t seed,
                                           ncsim_circuit** out);
/* Trajectory t: StdRng::seed_from_u64(seed0 + t), n = n_lo + gen_range(0..n_span),
 * the random-layer circuit of `depth` layers with DEPOLARIZE2(p) after every
 * CZ and M on every qubit (ncsim_workload_random_circuit_rng), run with the
 * same generator. */
ncsim_status ncsim_batch_random_layers(uint32_t count, uint64_t seed0, uint32_t n_lo, uint32_t n_span, uint32_t depth,
                                       double p, ncsim_batch** out);
#ifdef __cplusplus
}
#endif

#endif /* NCSIM_WORKLOADS_H */
