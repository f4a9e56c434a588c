// Launchers shared between the overlap_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace ovl {

struct Lattice;

constexpr int kSitesPerCta = 8;  // sites per CTA of the Wilson kernels (8 warps)

// Wilson operator on mode blocks [mb_first, mb_first + n_mb) of src.
// accumulate: dst(+same offset) += dt * D src; otherwise dst (a buffer of
// n_mb blocks) = D src.
template <typename T>
void launch_wilson(const double *links, const void *src, void *dst, const Lattice &L, int mb_first, int n_mb,
                   double amass, double dt, bool accumulate, cudaStream_t stream);
template <typename T>
void launch_axpy(void *dst, const void *deriv, size_t n_complex, double dt, int sm_count, cudaStream_t stream);

// Gauge fields (FP64).
void launch_update_links(double *U, const double *E, const Lattice &L, double dt_step, cudaStream_t stream);
void launch_update_efield(const double *U, double *E, double *dE, const Lattice &L, double dt_step, cudaStream_t stream);

// Reductions.  partial: caller-provided device scratch of reduce_partial_doubles()
// doubles; out: device array of the result size.
size_t ncsdot_partial_doubles(const Lattice &L);
void launch_ncsdot(const double *U, const double *E, const Lattice &L, double *partial, double *out, cudaStream_t stream);
size_t bulk_partial_doubles(const Lattice &L);
void launch_bulk(const double *U, const double *E, const Lattice &L, double *partial, double *out, cudaStream_t stream);

// Currents: 16 doubles per site (jV[4], jA[4], jVw[4], jAw[4]) + PS + WA = 18.
constexpr int kCurrentsPerSite = 18;
int currents_groups(int n_mb);
size_t currents_partial_doubles(const Lattice &L, int n_mb);
template <typename T>
void launch_currents(const double *U, const void *psi, const Lattice &L, int n_mb, int n_modes, int first_mode,
                     double r_wilson, double *partial, double *per_site, cudaStream_t stream);
void launch_site_sums(const double *per_site, const Lattice &L, double *partial, double *out4, cudaStream_t stream);

// Layout conversion between the reference layout (double, [mode][site][comp])
// and the mode-block layout of precision T.  Modes [m0, m0+count).
template <typename T>
void launch_ref_to_blocks(const double *ref, void *blocks, const Lattice &L, int m0, int count, cudaStream_t stream);
template <typename T>
void launch_blocks_to_ref(const void *blocks, double *ref, const Lattice &L, int m0, int count, cudaStream_t stream);

// Free Wilson plane waves for local modes [0, n_modes) (global index first_mode + m).
template <typename T>
void launch_free_fermions(void *psi, void *psimid, const Lattice &L, int n_modes, int n_mb, int first_mode,
                          double r_wilson, double m_fermion, double dt, int *bad, cudaStream_t stream);

}  // namespace ovl
