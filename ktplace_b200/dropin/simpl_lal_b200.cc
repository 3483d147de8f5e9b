// Drop-in replacement for KTPlace's globalPlacer/simpl/simpl_lal.cc.
//
// Compiled against the reference's own header (globalPlacer/simpl/
// simpl_lal.h), it defines the one member the SimPL placer calls,
//
//   LookAheadLegalizer::legalize (reference: simpl_lal.cc:43-123, with the
//                                 helpers of :125-372) -> ktg_lal
//
// (called from simplPlacer::Impl::lookAheadLegalize, simpl_placer.cc:299-310),
// and runs it on a B200. Link this object instead of simpl_lal.o, next to
// simpl_lss_b200.o.
//
// The legalizer keeps its own GPU context (device $KTPLACE_B200_DEVICE,
// default 0) holding the cells' sizes as a netlist without nets, the bin grid
// and the free space; each is installed again only when the placer hands over
// a different one (the refinement phase rebuilds the grid at a finer size).
// The positions are the reference legalizer's, bit for bit, when the cell
// areas are exact binary fractions (integer site areas are). Errors from the
// GPU are fatal through ktlog, as the reference treats its own unrecoverable
// states.
#include "globalPlacer/simpl/simpl_lal.h"
#include "util/kt_log.h"

#include "ktplace_b200.h"

#include <cstdint>
#include <cstdlib>
#include <vector>

namespace ktplace::simpl {
namespace {

struct LalGpu {
    ktg_ctx *ctx = nullptr;
    // what is installed
    const double *width = nullptr, *height = nullptr;
    std::size_t cells = ~std::size_t{0};
    const BinGrid *grid = nullptr;
    const double *avail = nullptr;
    std::size_t bins = 0;
    double density = -1.0;
    const FreeSpace *freeSpace = nullptr;
    std::size_t rows = 0;
    const std::vector<BBox> *obstacles = nullptr;
    std::size_t numObstacles = 0;
};

LalGpu &lalGpu() {
    static LalGpu s;
    return s;
}

void check(const char *what, int rc) {
    if (rc != KTG_OK) {
        const ktg_ctx *c = lalGpu().ctx;
        ktlog.fatal("ktplace_b200: {} failed ({}): {}", what, rc, c ? ktg_last_error(c) : "");
    }
}

// The cells as a netlist without nets: vertex i is movable cell i.
void installCells(LalGpu &s, const std::vector<double> &width, const std::vector<double> &height) {
    const std::size_t n = width.size();
    std::vector<int32_t> ids(n);
    for (std::size_t i = 0; i < n; ++i) ids[i] = static_cast<int32_t>(i);
    std::vector<double> zeros(n, 0.0);
    std::vector<int64_t> pinStart(n + 1, 0), netStart(1, 0);
    const ktg_netlist_view view{static_cast<int64_t>(n), static_cast<int64_t>(n), 0,
                                ids.data(), ids.data(), zeros.data(), zeros.data(),
                                netStart.data(), nullptr, nullptr, nullptr, nullptr,
                                pinStart.data(), nullptr, nullptr, width.data(), height.data()};
    check("ktg_upload_netlist", ktg_upload_netlist(s.ctx, &view));
    s.width = width.data();
    s.height = height.data();
    s.cells = n;
}

}  // namespace

void LookAheadLegalizer::legalize(std::vector<double> &x, std::vector<double> &y) const {
    LalGpu &s = lalGpu();
    if (s.ctx == nullptr) {
        const char *dev = std::getenv("KTPLACE_B200_DEVICE");
        check("ktg_create", ktg_create(dev ? std::atoi(dev) : 0, &s.ctx));
    }
    if (s.width != width.data() || s.height != height.data() || s.cells != width.size())
        installCells(s, width, height);
    if (s.grid != &grid || s.avail != grid.avail.data() || s.bins != grid.size() ||
        s.density != densityLimit) {
        const ktg_grid_view g{grid.origin.x, grid.origin.y, grid.dx, grid.dy,
                              static_cast<int64_t>(grid.nx), static_cast<int64_t>(grid.ny),
                              grid.avail.data(), grid.totalAvail, densityLimit};
        check("ktg_set_grid", ktg_set_grid(s.ctx, &g));
        s.grid = &grid;
        s.avail = grid.avail.data();
        s.bins = grid.size();
        s.density = densityLimit;
    }
    if (s.freeSpace != &freeSpace || s.rows != freeSpace.rows.size() || s.obstacles != &obstacles ||
        s.numObstacles != obstacles.size()) {
        std::vector<double> rowY, spans, obst;
        std::vector<int64_t> rowSpan(1, 0);
        for (const FreeSpace::Row &r : freeSpace.rows) {
            rowY.push_back(r.y.start);
            rowY.push_back(r.y.end);
            for (const Interval &sp : r.spans) {
                spans.push_back(sp.start);
                spans.push_back(sp.end);
            }
            rowSpan.push_back(static_cast<int64_t>(spans.size() / 2));
        }
        for (const BBox &o : obstacles) {
            obst.push_back(o.lowerLeft.x);
            obst.push_back(o.lowerLeft.y);
            obst.push_back(o.upperRight.x);
            obst.push_back(o.upperRight.y);
        }
        const double dieBox[4] = {die.lowerLeft.x, die.lowerLeft.y, die.upperRight.x,
                                  die.upperRight.y};
        check("ktg_set_free_space",
              ktg_set_free_space(s.ctx, static_cast<int64_t>(freeSpace.rows.size()), rowY.data(),
                                 rowSpan.data(), spans.data(),
                                 static_cast<int64_t>(obstacles.size()), obst.data(), dieBox));
        s.freeSpace = &freeSpace;
        s.rows = freeSpace.rows.size();
        s.obstacles = &obstacles;
        s.numObstacles = obstacles.size();
    }
    check("ktg_lal", ktg_lal(s.ctx, x.data(), y.data(), static_cast<int32_t>(opts.maxLevel),
                             static_cast<int32_t>(opts.minCellsToSplit), opts.stripeAreaFraction));
}

}  // namespace ktplace::simpl
