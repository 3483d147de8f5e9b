// GPU bodies for two private members of KTPlace's simplPlacer::Impl
// (globalPlacer/simpl/simpl_placer.cc:256-289), for a simpl_placer.cc whose
// two member bodies are replaced by calls to them (oracle/hooks/
// apply_hooks.py writes such a copy): getHpwl -> ktg_hpwl, getOccupancy ->
// ktg_occupancy; getOverflow keeps its host loop over the returned map. They run on the
// same GPU context as the drop-in's buildB2B / solveBothAxes
// (simpl_lss_b200.cc), which then holds the cells' real sizes.
#pragma once

#include <vector>

#include "globalPlacer/simpl/simpl_grid.h"
#include "globalPlacer/simpl/simpl_lss.h"

namespace ktplace::simpl::b200 {

// simplPlacer::Impl::getHpwl (simpl_placer.cc:256-275): the per-net half
// perimeters summed in the reference's order (ktg option "hpwl_order" 2,
// unless $KTPLACE_B200_HPWL_ORDER=0), so the value is bit-identical.
double hpwl(const Netlist &netlist, const std::vector<double> &x, const std::vector<double> &y);

// simplPlacer::Impl::getOccupancy (simpl_placer.cc:282-289): the movable
// area of every bin of `grid`, binned at the cells' centres (64-bit fixed
// point on the device; bit-identical when the areas are dyadic, such as
// integer site areas). The grid is installed on the device when it changes.
std::vector<double> occupancy(const Netlist &netlist, const std::vector<double> &width,
                              const std::vector<double> &height, const BinGrid &grid,
                              double densityLimit, const std::vector<double> &x,
                              const std::vector<double> &y);

}  // namespace ktplace::simpl::b200
