// coupling.cu -- CFD-DEM coupling entry points (drag and mean fields).
#include "dem_internal.cuh"

using namespace demb;


extern "C" {
int dem_set_gas_fields(dem_handle* h, const dem_fluid_grid*, const double*, const double*, const double*,
                       const double*, const double*) {
  return set_err(h, DEM_ERR_STATE, "coupling not built");
}
int dem_get_mean_fields(dem_handle* h, double*, double*) { return set_err(h, DEM_ERR_STATE, "coupling not built"); }
int dem_comp_mean_fields(dem_handle* h) { return set_err(h, DEM_ERR_STATE, "coupling not built"); }
int dem_drag_gs_des0(dem_handle* h) { return set_err(h, DEM_ERR_STATE, "coupling not built"); }
int dem_step_coupled(dem_handle* h, int32_t, int32_t) { return set_err(h, DEM_ERR_STATE, "coupling not built"); }
}
