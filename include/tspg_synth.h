/*
 * tspg_synth.h — seeded synthetic operands of the benchmark workloads and the
 * .bmtx fixture reader (host code, libtspg_synth.so).
 *
 * Kept apart from the device library (libtspg.so, include/tspg.h) so that a
 * CPU-only consumer — the timed CPU baseline of the benchmark — builds the same
 * matrices without mapping the GPU product.  Every random draw comes from a
 * counter-based generator (splitmix64 of seed, stream and counter), so a matrix
 * depends only on its parameters and seed, never on the thread count.
 * Status codes are the TSPG_* codes of tspg.h.
 */
#ifndef TSPG_SYNTH_H
#define TSPG_SYNTH_H

#include <stddef.h>
#include <stdint.h>

#include "tspg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Host CSR with int64 row offsets and FP64 values.  Arrays are allocated with
 * malloc and released with tspg_host_free. */
typedef struct tspg_host_csr {
  int64_t nrows, ncols, nnz;
  int64_t *rowptr;
  int32_t *col;
  double *val;
} tspg_host_csr;
void tspg_host_free(tspg_host_csr *M);
/* n x n, row i = k distinct uniform columns plus (if diag) column i. */
int tspg_gen_uniform_rows(int64_t n, int k, int diag, uint64_t seed,
                          tspg_host_csr *out);
/* R-MAT: 2^scale rows, edge_factor*2^scale draws, quadrant probabilities
 * a, b, c (d = 1-a-b-c), duplicates merged, self-loops kept. */
int tspg_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                  uint64_t seed, tspg_host_csr *out);
/* 27-point (pts=27, 26 / -1) or 7-point (pts=7, 6 / -1) Laplacian on an
 * nx*ny*nz grid, lexicographic x-fastest numbering. */
int tspg_gen_laplacian(int64_t nx, int64_t ny, int64_t nz, int pts,
                       tspg_host_csr *out);
/* Smoothed-aggregation prolongator P = (I - omega D^-1 A) P_tent for a
 * Laplacian A from tspg_gen_laplacian, aggregates agg^3 by integer division
 * of the grid coordinates, P_tent 0/1 (unnormalised). */
int tspg_gen_sa_prolongator(int64_t nx, int64_t ny, int64_t nz, int pts,
                            int agg, double omega, tspg_host_csr *out);
/* Host transpose (R = P^T for the Galerkin product). */
int tspg_host_transpose(const tspg_host_csr *M, tspg_host_csr *out);
/* Random square matrix of the batched workload: rows x rows, row lengths
 * Poisson(lambda), distinct uniform columns. */
int tspg_gen_poisson_rows(int64_t rows, double lambda, uint64_t seed,
                          tspg_host_csr *out);
/* Read a Trident .bmtx file (MatrixMarket banner with index and value byte
 * widths, then little-endian (row, col, float32) records) into CSR with
 * duplicates kept in file order. */
int tspg_read_bmtx(const char *path, tspg_host_csr *out);

#ifdef __cplusplus
}
#endif
#endif /* TSPG_SYNTH_H */
