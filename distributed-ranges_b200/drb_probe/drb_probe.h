/*
 * drb_probe.h -- the streaming-gather probe (measurement only).
 *
 * No counterpart in the reference, and not part of the product's C ABI
 * (include/drb.h): lib/libdrb_probe.so exports it for the bench, which
 * times it beside the SpMV as the floor of a gather-bound product.
 */
#ifndef DRB_PROBE_H
#define DRB_PROBE_H

#include "drb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Streams A's column indices (and its values when with_values != 0) with the
 * SpMV's 16-byte loads and gathers x[col] at every nonzero: the reads of
 * y = A x without rows, row sums or y, so its time is a floor for any SpMV on
 * this pattern that fetches x element by element (random columns make that,
 * not HBM, the bound).  Writes nothing the caller sees.  F32 or F64 storage
 * (else DRB_ERR_UNSUPPORTED); x: device, n elements of the value type. */
drb_status drb_csr_gather_probe(drb_csr_t A, const void *x, int with_values,
                                void *stream);

/* The k right-hand-side form: X row-major (n rows of ldx elements, 16-byte
 * aligned); every nonzero gathers its whole X row of k elements in 16-byte
 * vectors while the column indices (and values) stream in nonzero order --
 * the reads of Y = A X without rows, sums or Y.  When X is far larger than
 * L2 both this and the SpMM are bound by random row reads from HBM, and the
 * SpMM's row-ordered items run a little faster than this plain stream, so it
 * is a reference rate, not a floor.  k * element size must be 16, 32, ...,
 * 512 bytes (a power of two) and ldx * element size a multiple of 16 (else
 * DRB_ERR_UNSUPPORTED).  F32 or F64 storage. */
drb_status drb_csr_gather_rows_probe(drb_csr_t A, const void *X, int64_t ldx, int64_t k,
                                     int with_values, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DRB_PROBE_H */
