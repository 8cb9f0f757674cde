// Host-side shim around the reference's exact element action (solver/src/materials/fi_modal.cuh).
// TEST INFRASTRUCTURE ONLY: built by oracle/Makefile into oracle/_ref/ straight from the header
// where it lies in the reference tree; nothing from the reference is copied into this repository.
// It exposes one C entry point that applies the element action to a batch of elements, so the
// oracle's dense Ke product can be checked against the reference arithmetic.
#define __device__
#define __forceinline__ inline
#include "fi_modal.cuh"

extern "C" void ref_fi_modal_batch(const double* u, const double* c21, const double* g, double* f, long count) {
  for (long e = 0; e < count; ++e) fi_modal(u + 24 * e, c21, 0.0, g, f + 24 * e);
}
