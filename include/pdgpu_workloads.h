/*
 * pdgpu_workloads.h -- host-side synthetic workload generators of libpdgpu.so
 * (no counterpart in the reference; its performance tests draw their own
 * synthetic particle sets, e.g. Vector/performance/vector_dist_performance_common.hpp:141-198).
 */
#ifndef PDGPU_WORKLOADS_H
#define PDGPU_WORKLOADS_H

#ifdef __cplusplus
extern "C" {
#endif

/* n particles in n_clusters Gaussian clusters (std sigma_c per axis) at uniform
 * centres in the periodic box [0, L)^3, no two closer than min_dist (minimum
 * image); a particle redrawn max_tries times moves its cluster's centre.
 * x_out: n x 3 (AoS).  centre_redraws (optional): number of centre moves. */
int pd_gen_clustered(long n, double L, int n_clusters, double sigma_c, double min_dist, unsigned long seed,
                     int max_tries, double* x_out, long* centre_redraws);

#ifdef __cplusplus
}
#endif
#endif /* PDGPU_WORKLOADS_H */
