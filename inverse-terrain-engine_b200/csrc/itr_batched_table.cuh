// itr_batched_table.cuh — the instantiations of k_batched for one (CREST, BND) pair.
//
// k_batched has 128 instantiations: crest faces, stage/inflow ghosts, cluster use, four block
// size buckets, locked dt and dry-row skipping. Each of the translation units itr_kb_<c><b>.cu
// instantiates the 32 of one (CREST, BND) pair through ITR_BATCHED_TABLE, so the library
// compiles in parallel; the self-checking build (-DITR_CHECKED) instantiates all four pairs
// in itr_capi.cu, one translation unit, so its error record g_itr_err is a single array.
#pragma once
#include "itr_batched.cuh"

namespace itr {

typedef void (*BatchedFn)(const BatchArgs);

template <bool CR, bool CL, bool BD, bool LK, bool SK>
BatchedFn batched_by_maxt(int maxt) {
  if (maxt <= 256) return k_batched<CR, CL, 256, BD, LK, SK>;
  if (maxt <= 512) return k_batched<CR, CL, 512, BD, LK, SK>;
  if (maxt <= 768) return k_batched<CR, CL, 768, BD, LK, SK>;
  return k_batched<CR, CL, 1024, BD, LK, SK>;
}

template <bool CR, bool BD>
BatchedFn batched_table(bool clustered, int maxt, bool locked, bool skip) {
  if (clustered) {
    if (locked) return skip ? batched_by_maxt<CR, true, BD, true, true>(maxt) : batched_by_maxt<CR, true, BD, true, false>(maxt);
    return skip ? batched_by_maxt<CR, true, BD, false, true>(maxt) : batched_by_maxt<CR, true, BD, false, false>(maxt);
  }
  if (locked) return skip ? batched_by_maxt<CR, false, BD, true, true>(maxt) : batched_by_maxt<CR, false, BD, true, false>(maxt);
  return skip ? batched_by_maxt<CR, false, BD, false, true>(maxt) : batched_by_maxt<CR, false, BD, false, false>(maxt);
}

// The kernel of (crest, bnd) = (C, B) for the remaining switches; one definition per pair.
BatchedFn batched_fn_00(bool clustered, int maxt, bool locked, bool skip);
BatchedFn batched_fn_01(bool clustered, int maxt, bool locked, bool skip);
BatchedFn batched_fn_10(bool clustered, int maxt, bool locked, bool skip);
BatchedFn batched_fn_11(bool clustered, int maxt, bool locked, bool skip);

#define ITR_BATCHED_TABLE(NAME, CR, BD)                                   \
  BatchedFn NAME(bool clustered, int maxt, bool locked, bool skip) {      \
    return batched_table<CR, BD>(clustered, maxt, locked, skip);          \
  }

}  // namespace itr
