// fe_tile_c16.cu -- solve drivers instantiated for column tiles of width 16.
#include "fe_solve_impl.cuh"

namespace fe {
template int solve_tile_C<16>(fe_plan*, const SolveReq&, int64_t, int, std::vector<Inst>&);
}  // namespace fe
