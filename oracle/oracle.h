/*
 * oracle.h — CPU restatement of Trident's on-node compute semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load this library, and
 * only as the checker or the timed CPU baseline; the product (libtspg) never
 * links or calls it.
 *
 * Pinning.
 *   - Bitmask gen / AND / pack / unpack: pinned to the known answers of the
 *     reference's own test (test/test_compression.cu:106-238, 550-590),
 *     restated in tests/golden/kat_bitmask.json.
 *   - SpGEMM and merge: parity unpinned at the library boundary.  The
 *     reference's local multiply is KokkosKernels 4.7.01 (a non-vendored
 *     submodule) and cuSPARSE; neither can run here, and the reference ships
 *     no outputs for its .bmtx fixtures.  The restatement follows the
 *     semantics the reference relies on (structural product, zeros kept,
 *     union merge) and is cross-checked in tests against dense products and
 *     scipy values.
 *
 * All row offsets here are int64, values FP64 (the pack takes raw value
 * bytes of any width).  Rows produced are sorted by column.
 */
#ifndef TSPG_ORACLE_H
#define TSPG_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

int orc_num_threads(void);
void orc_set_threads(int n);

/* mults per row i in [r0, r1) (written to row_mults[i - r0] when non-NULL);
 * returns the sum.  KokkosSparse::spgemm / cusparseSpGEMM_getNumProducts
 * (include/cusparse_helpers.cuh:981-985). */
int64_t orc_row_mults(int64_t r0, int64_t r1, const int64_t *Ap,
                      const int32_t *Aj, const int64_t *Bp,
                      int64_t *row_mults);

/* Row counts of C = A·B for rows [r0, r1) (structural: (i,j) in C iff some k
 * has A_ik and B_kj stored).  Writes cnt[i - r0]; returns the sum. */
int64_t orc_spgemm_count(int64_t r0, int64_t r1, int64_t ncols,
                         const int64_t *Ap, const int32_t *Aj,
                         const int64_t *Bp, const int32_t *Bj, int64_t *cnt);

/* Numeric C = A·B for rows [r0, r1): writes row i at Cj/Cx + Cp[i] - Cp[r0],
 * sorted by column.  Accumulates in FP64 in A-row order then B-row order.
 * When Cabs is non-NULL it also receives sum |a_ik * b_kj| per entry (the
 * scale for the 1e-12 value tolerance). */
int orc_spgemm_numeric(int64_t r0, int64_t r1, int64_t ncols,
                       const int64_t *Ap, const int32_t *Aj, const double *Ax,
                       const int64_t *Bp, const int32_t *Bj, const double *Bx,
                       const int64_t *Cp, int32_t *Cj, double *Cx,
                       double *Cabs);

/* Union merge C = A + B of sorted, duplicate-free rows
 * (cusparse_spgeam, include/cusparse_helpers.cuh:799-905). */
int64_t orc_spadd_count(int64_t m, const int64_t *Ap, const int32_t *Aj,
                        const int64_t *Bp, const int32_t *Bj, int64_t *cnt);
int orc_spadd_numeric(int64_t m, const int64_t *Ap, const int32_t *Aj,
                      const double *Ax, const int64_t *Bp, const int32_t *Bj,
                      const double *Bx, const int64_t *Cp, int32_t *Cj,
                      double *Cx);

/* SpaComm::gen_bitmask (include/spacomm.cuh:29-117): n segments of ptr,
 * ceil(n/8) bytes, bit (i % 8) of byte i/8 set iff ptr[i] != ptr[i+1]. */
void orc_bitmask_gen(const int64_t *ptr, int64_t n, uint8_t *out);
/* SpaComm::intersect_bitmasks (include/spacomm.cuh:126-148). */
void orc_bitmask_and(const uint8_t *a, const uint8_t *b, int64_t nbytes,
                     uint8_t *out);
/* select_entries (include/spacomm.cuh:428-537, keep rule :714-782) plus
 * select_ptrs (:556-623) on one tile: ptr has len+1 entries; idx/val hold
 * ptr[len] entries of val_bytes each.  Writes the kept entries in order and
 * the full-length packed ptr; returns the kept count. */
int64_t orc_pack(const int64_t *ptr, int64_t len, const int32_t *idx,
                 const void *val, int val_bytes, const uint8_t *mask,
                 int64_t *out_ptr, int32_t *out_idx, void *out_val);

#ifdef __cplusplus
}
#endif
#endif
