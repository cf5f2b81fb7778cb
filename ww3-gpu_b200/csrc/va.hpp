// ww3-gpu_b200/csrc/va.hpp
// The resident spectrum: VA(NSPEC, 0:NSEALM) of one WW3 grid kept in HBM for the whole run,
// beside the Fortran array it mirrors, with a state saying which copy holds the newer bits.
//
// Reference: ww3-gpu kokkos/src/ww_kokkos/resident_state.hpp:15-40 and
// kokkos/src/fortran_iface/resident_shim.cpp (the ww_va_* protocol of resident_c.hpp:1-101):
// bind on the first call, refuse another address or shape, copy whole arrays only when the
// other side is newer, partial reads/writes of listed columns that leave the state alone, and
// the WW_KOKKOS_VA_RESIDENT / _CHECK / _POISON / _COUNT diagnostics.
//
// Layout in HBM: d_va is the Fortran array's bytes, column-major, column JSEA (0..NSEALM) of
// NSPEC floats at d_va + JSEA*NSPEC; column 0 is WW3's sink column.
#pragma once

#include <cstddef>

namespace wwb {

/// The device copy of grid `igrid`'s VA, holding the newer bits: binds `va` on the grid's first
/// call, refuses another address or shape (BAD_SHAPE), copies host to device when the host is
/// newer. Returns a WwKokkosStatus.
int va_device(int igrid, float* va, int nspec, int nsealm, float** d_va);

/// After a kernel wrote d_va of `igrid`: the device holds the newer bits.
void va_device_written(int igrid);

/// Before launches that read and write a bound grid's d_va without naming the host array (a
/// recorded step): uploads the host copy when it is the newer one. An unbound grid is left
/// alone. Returns a WwKokkosStatus.
int va_device_current(int igrid);

/// Frees every grid's device copy (ww_kokkos_finalize).
void release_va_contexts();

}  // namespace wwb
