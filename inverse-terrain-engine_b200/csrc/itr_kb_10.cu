// k_batched instantiations with crest faces on and stage/inflow ghosts off
// (one of four translation units, itr_batched_table.cuh).
#ifndef ITR_CHECKED
#include "itr_batched_table.cuh"
namespace itr {
ITR_BATCHED_TABLE(batched_fn_10, true, false)
}  // namespace itr
#endif
