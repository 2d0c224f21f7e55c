/*
 * wilson_probe.h -- integer-pipe microbenchmarks of libwilson.so.
 *
 * No counterpart in the reference: these measure the GPU's integer multiply
 * throughput on the box, which is the roofline of the column sweep (the
 * reference's kernels are integer-multiply bound too, kernels/common.cl:41-67).
 */
#ifndef WILSON_PROBE_H
#define WILSON_PROBE_H

#ifdef __cplusplus
extern "C" {
#endif

#define WL_PROBE_MAD    0   /* mad.lo.u32 operations per second */
#define WL_PROBE_MADHI  1   /* mad.hi.u32 operations per second */
#define WL_PROBE_CELL2  2   /* sweep cells per second, 2-limb residues (p < 2^31) */
#define WL_PROBE_CELL3  3   /* sweep cells per second, 3-limb residues (p < 2^47) */
#define WL_PROBE_CELL4  4   /* sweep cells per second, 4-limb residues (p < 2^62) */
#define WL_PROBE_MADWIDE 5  /* mad.wide.u32 operations per second */
/* 100 + 10*(L-2) + v: cell formulation v (0 carry-flag chain, 1 wide
   products, 2 wide products with a high-half first reduction) at width L */

/* Run one microbenchmark on `device`; *rate receives operations (or cells) per second. */
int wl_probe(int device, int which, double *rate);

#ifdef __cplusplus
}
#endif

#endif /* WILSON_PROBE_H */
