/*
 * Numerical-spacetime kernels (interp.cl + dyst.cl).  Filled in by the
 * numerical-spacetime milestone; until then every entry reports
 * cudaErrorNotSupported so the C ABI returns GRAY_ECUDA loudly.
 */
#include "gray_internal.h"

cudaError_t
launch_dyst_icond(const RenderParams &, const GridParams &, double *, double *, cudaStream_t)
{
	return cudaErrorNotSupported;
}

cudaError_t
launch_dyst_evolve64(const RenderParams &, const GridParams &, double *, double *, double,
                     long long, unsigned long long *, cudaStream_t)
{
	return cudaErrorNotSupported;
}

cudaError_t
launch_dyst_mixed(const RenderParams &, const GridParams &, double *, double *, double, double,
                  long long, long long, unsigned long long *, unsigned int *, cudaStream_t,
                  const MixedLaunch &)
{
	return cudaErrorNotSupported;
}

cudaError_t
launch_boosted_ks(const GridParams &, float *, double, double, int, double, cudaStream_t)
{
	return cudaErrorNotSupported;
}
