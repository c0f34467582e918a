// k_batched instantiations with crest faces off and stage/inflow ghosts on
// (one of four translation units, itr_batched_table.cuh).
#ifndef ITR_CHECKED
#include "itr_batched_table.cuh"
namespace itr {
ITR_BATCHED_TABLE(batched_fn_01, false, true)
}  // namespace itr
#endif
