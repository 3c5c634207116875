// read.h -- read-out kernel launchers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ket_sv.h"

namespace ket {

#define KET_MAX_MARGINAL_QUBITS 12
#define KET_PAULI_GROUP_TERMS 64

struct MarginalSpec {
  int m;
  int q[KET_MAX_MARGINAL_QUBITS];
  uint64_t mask;
};

struct PauliGroup {
  uint64_t flip;                        // X|Y positions
  int ny;                               // number of Y factors (mod 4 phase i^ny)
  int nterms;
  uint64_t zm[KET_PAULI_GROUP_TERMS];   // Z|Y positions of each term
  double coeff[KET_PAULI_GROUP_TERMS];
};

int num_sms();

cudaError_t launch_norm2(const void* amp, int n, int prec, double* scratch, double* out, cudaStream_t s);
size_t norm2_scratch(int n);
cudaError_t launch_probs_dense(const void* amp, int prec, uint64_t off, uint64_t cnt, double thr, double* out,
                               cudaStream_t s);
uint64_t kept_chunk(int n);
cudaError_t launch_count_kept(const void* amp, int n, int prec, double thr, uint64_t* counts, cudaStream_t s);
cudaError_t launch_compact_kept(const void* amp, int n, int prec, double thr, const uint64_t* offs, uint64_t cap,
                                uint64_t* oidx, double* op, cudaStream_t s);
uint64_t marg_chunk(int n);
cudaError_t launch_marginals(const void* amp, int n, int prec, double* partial, double* out, cudaStream_t s);
int mdist_chunk_bits(int n, int m);
cudaError_t launch_marginal_dist(const void* amp, int n, int prec, const MarginalSpec& spec, double* partial,
                                 double* out, cudaStream_t s);
// Sampling: the reference's running FP64 sum over kept entries in ascending
// index order, bit for bit, kept as one checkpoint per 32 entries; each draw
// (0 <= r <= 1) searches the checkpoints and adds inside one sub-chunk.
size_t sample_scratch(int n);
int sample_launches();
cudaError_t launch_sample(const void* amp, int n, int prec, double thr, const double* r, uint64_t shots, void* scratch,
                          uint64_t* out, cudaStream_t s);
cudaError_t launch_gather(const void* amp, int prec, const uint64_t* idx, uint64_t k, double* out, cudaStream_t s);
cudaError_t launch_pauli_group(const void* amp, int n, int prec, const PauliGroup& g, double* partial, double* out,
                               cudaStream_t s);
size_t pauli_scratch(int n);

// <a|b> (re, im) and max |a_i - b_i| of two states of the same size, any precisions.
cudaError_t launch_compare(const void* a, int pa, const void* b, int pb, int n, double* scratch, double* out,
                           cudaStream_t s);
size_t compare_scratch(int n);

}  // namespace ket
