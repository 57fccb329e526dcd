// fe_tile_c4.cu -- solve drivers instantiated for column tiles of width 4.
#include "fe_solve_impl.cuh"

namespace fe {
template int solve_tile_C<4>(fe_plan*, const SolveReq&, int64_t, int, std::vector<Inst>&);
}  // namespace fe
