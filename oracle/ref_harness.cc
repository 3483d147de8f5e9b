// Oracle harness around the reference's own SimPL code (test infrastructure).
//
// This translation unit is compiled against the reference sources where they
// lie (see oracle/Makefile) and linked with the reference's own compiled
// simpl_lss.cc, simpl_lal.cc, simpl_dm.cc, datamodel/, util/, geometry/ and
// adaptor/ objects plus the project TBB shim. It adds nothing to the algorithm:
// every number it returns is computed by reference code.
//
//   * ref_build_b2b   -> LinearSystems::buildB2B    (simpl_lss.cc:11-114)
//   * ref_build_star  -> LinearSystems::buildStar   (simpl_lss.cc:116-201)
//   * ref_solve       -> solveBothAxes             (simpl_lss.cc:203-290)
//   * ref_hpwl        -> simplPlacer::Impl::getHpwl (simpl_placer.cc:256-275)
//   * ref_occupancy   -> Impl::getOccupancy + getOverflow (simpl_placer.cc:282-297)
//   * ref_grid        -> Impl::buildGrid            (simpl_placer.cc:190-224)
//   * ref_floors      -> Impl::collect              (simpl_placer.cc:169-179)
//   * ref_lal         -> Impl::lookAheadLegalize (simpl_placer.cc:299-310,
//                        LookAheadLegalizer::legalize, simpl_lal.cc:43-123)
//   * ref_free_space  -> the FreeSpace rows Impl::buildGrid made (simpl_grid.h:130-173)
//   * ref_design_load_bookshelf -> BookshelfInputAdapter + buildSimplDM
//     (adaptor/bookshelfToKTAdaptor.cc, simpl_dm.cc:16-85,262-279)
//
// The Impl members are private to simpl_placer.cc, so that file is included
// here (it is not linked separately) and its members are reached through the
// explicit-instantiation access rule ([temp.spec.general]: access checking is
// not applied to names in an explicit instantiation).
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg load the shared
// library built from this file; the CUDA product never does.

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <exception>
#include <iostream>
#include <memory>
#include <string>
#include <string_view>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "adaptor/kt_inputReader.h"
#include "datamodel/kt_dm.h"
#include "globalPlacer/simpl/simpl_dm.h"
#include "globalPlacer/simpl/simpl_lss.h"
#include "util/kt_log.h"

#include "globalPlacer/simpl/simpl_placer.cc"

namespace {

using namespace ktplace;
using namespace ktplace::simpl;

// ---- explicit-instantiation access to simplPlacer's private pieces ----------
template <typename Tag, auto Member>
struct Grant {
    friend auto reach(Tag) { return Member; }
};

struct PImplTag { friend auto reach(PImplTag); };
struct CollectTag { friend auto reach(CollectTag); };
struct BuildGridTag { friend auto reach(BuildGridTag); };
struct HpwlTag { friend auto reach(HpwlTag); };
struct OccTag { friend auto reach(OccTag); };
struct OverflowTag { friend auto reach(OverflowTag); };
struct DensityTag { friend auto reach(DensityTag); };
struct GridTag { friend auto reach(GridTag); };
struct FloorXTag { friend auto reach(FloorXTag); };
struct FloorYTag { friend auto reach(FloorYTag); };
struct DieTag { friend auto reach(DieTag); };
struct LalTag { friend auto reach(LalTag); };
struct FreeTag { friend auto reach(FreeTag); };

}  // namespace

template struct Grant<PImplTag, &simplPlacer::pImpl>;
template struct Grant<CollectTag, &simplPlacer::Impl::collect>;
template struct Grant<BuildGridTag, &simplPlacer::Impl::buildGrid>;
template struct Grant<HpwlTag, &simplPlacer::Impl::getHpwl>;
template struct Grant<OccTag, &simplPlacer::Impl::getOccupancy>;
template struct Grant<OverflowTag, &simplPlacer::Impl::getOverflow>;
template struct Grant<DensityTag, &simplPlacer::Impl::densityLimit>;
template struct Grant<GridTag, &simplPlacer::Impl::grid>;
template struct Grant<FloorXTag, &simplPlacer::Impl::floorX>;
template struct Grant<FloorYTag, &simplPlacer::Impl::floorY>;
template struct Grant<DieTag, &simplPlacer::Impl::die>;
template struct Grant<LalTag, &simplPlacer::Impl::lookAheadLegalize>;
template struct Grant<FreeTag, &simplPlacer::Impl::freeSpace>;

namespace {

struct Handle {
    std::unique_ptr<ktDM> db;       // kept alive when loaded from Bookshelf
    Design design;                  // SimPL's flattened design
    std::unique_ptr<simplPlacer> placer;
    SparseSystem sysX;
    SparseSystem sysY;
    std::string error;

    auto &impl() { return *((*placer).*reach(PImplTag{})); }
    void attach() {
        placer = std::make_unique<simplPlacer>(design);
        auto &im = impl();
        (im.*reach(CollectTag{}))();
        im.*reach(DieTag{}) = design.die;
    }
};

std::streambuf *savedCerr = nullptr;

// The reference logger echoes banners and tables on std::cerr; the harness
// mutes it (fatal messages still surface as exceptions).
void setQuiet(bool on) {
    if (on && savedCerr == nullptr) {
        savedCerr = std::cerr.rdbuf(nullptr);
    } else if (!on && savedCerr != nullptr) {
        std::cerr.rdbuf(savedCerr);
        std::cerr.clear();
        savedCerr = nullptr;
    }
}

void quiet() {
    static bool done = false;
    if (!done) {
        ktlog.throwOnFatal(true);
        setQuiet(true);
        done = true;
    }
}

template <typename F>
int guarded(Handle *h, F &&f) {
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        if (h != nullptr) h->error = e.what();
        return -1;
    }
}

}  // namespace

extern "C" {

void ref_set_quiet(int on) { setQuiet(on != 0); }

int ref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

const char *ref_last_error(void *hp) {
    return hp ? static_cast<Handle *>(hp)->error.c_str() : "null handle";
}

// Reads a Bookshelf directory with the reference reader and flattens it with
// the reference's buildSimplDM. Returns nullptr on failure.
void *ref_design_load_bookshelf(const char *dir) {
    quiet();
    try {
        auto reader = makeInputReader(dir);
        if (!reader) return nullptr;
        auto h = std::make_unique<Handle>();
        h->db = reader->read(dir);
        if (!h->db) return nullptr;
        simplDM dm = buildSimplDM(*h->db);
        h->design = dm.getDesign();
        h->attach();
        return h.release();
    } catch (const std::exception &) {
        return nullptr;
    }
}

// Builds the SimPL design straight from flattened arrays (same meaning as the
// members of Netlist, simpl_lss.h:27-36). Rows are (coordinate, height, pitch,
// xlo, xhi) with one subrow each; obstacles are (lx, ly, ux, uy).
void *ref_design_from_arrays(uint64_t numVertices, uint64_t numMovable, const uint32_t *movVertex,
                             const double *fixedX, const double *fixedY, uint64_t numNets,
                             const uint64_t *netStart, const uint32_t *pinCell, const double *offX,
                             const double *offY, const double *netWeight, const double *width,
                             const double *height, uint64_t numObstacles, const double *obstacles,
                             uint64_t numRows, const double *rows, const double *die4) {
    quiet();
    try {
        auto h = std::make_unique<Handle>();
        Design &d = h->design;
        Netlist &nl = d.netlist;
        nl.numMovable = numMovable;
        nl.movVertex.assign(movVertex, movVertex + numMovable);
        nl.varOfVertex.assign(numVertices, noVar);
        for (uint64_t i = 0; i < numMovable; ++i) nl.varOfVertex[movVertex[i]] = static_cast<uint32_t>(i);
        nl.fixedX.assign(fixedX, fixedX + numVertices);
        nl.fixedY.assign(fixedY, fixedY + numVertices);
        nl.nets.resize(numNets);
        for (uint64_t n = 0; n < numNets; ++n) {
            NetPins &np = nl.nets[n];
            np.weight = netWeight[n];
            for (uint64_t p = netStart[n]; p < netStart[n + 1]; ++p) {
                np.cells.push_back(pinCell[p]);
                np.offX.push_back(offX[p]);
                np.offY.push_back(offY[p]);
            }
        }
        // cell -> (net, pin) in ascending net order, as collectNets builds it.
        nl.pinStart.assign(numMovable + 1, 0);
        for (const NetPins &np : nl.nets)
            for (uint32_t c : np.cells)
                if (nl.varOfVertex[c] != noVar) ++nl.pinStart[nl.varOfVertex[c] + 1];
        for (uint64_t i = 0; i < numMovable; ++i) nl.pinStart[i + 1] += nl.pinStart[i];
        nl.pinsOfCell.resize(nl.pinStart.back());
        std::vector<std::size_t> cursor(nl.pinStart.begin(), nl.pinStart.end() - 1);
        for (uint32_t n = 0; n < nl.nets.size(); ++n)
            for (uint32_t q = 0; q < nl.nets[n].cells.size(); ++q) {
                const uint32_t v = nl.varOfVertex[nl.nets[n].cells[q]];
                if (v != noVar) nl.pinsOfCell[cursor[v]++] = {.net = n, .pin = q};
            }
        for (uint64_t i = 0; i < numMovable; ++i) {
            d.width.push_back(width[i]);
            d.height.push_back(height[i]);
            d.area.push_back(width[i] * height[i]);
            d.region.push_back(Fences::noRegion);
            d.x.push_back(0.0);
            d.y.push_back(0.0);
        }
        d.numFixed = numVertices - numMovable;
        for (uint64_t o = 0; o < numObstacles; ++o)
            d.obstacles.push_back(BBox(Point(obstacles[4 * o], obstacles[4 * o + 1]),
                                       Point(obstacles[4 * o + 2], obstacles[4 * o + 3])));
        for (uint64_t r = 0; r < numRows; ++r) {
            simpl::RowInfo ri{.coordinate = rows[5 * r], .height = rows[5 * r + 1],
                       .sitePitch = rows[5 * r + 2], .subrows = {}};
            ri.subrows.push_back(Subrow{.x = Interval(rows[5 * r + 3], rows[5 * r + 4])});
            d.rows.push_back(std::move(ri));
        }
        d.die = BBox(Point(die4[0], die4[1]), Point(die4[2], die4[3]));
        h->attach();
        return h.release();
    } catch (const std::exception &) {
        return nullptr;
    }
}

void ref_design_free(void *hp) { delete static_cast<Handle *>(hp); }

// sizes: V, n, N, P (deduplicated pins), P_mov (cell->pin refs), numFixed,
// numObstacles, numRows
int ref_netlist_sizes(void *hp, uint64_t *out) {
    auto *h = static_cast<Handle *>(hp);
    const Netlist &nl = h->design.netlist;
    uint64_t P = 0;
    for (const NetPins &np : nl.nets) P += np.cells.size();
    out[0] = nl.varOfVertex.size();
    out[1] = nl.numMovable;
    out[2] = nl.nets.size();
    out[3] = P;
    out[4] = nl.pinsOfCell.size();
    out[5] = h->design.numFixed;
    out[6] = h->design.obstacles.size();
    out[7] = h->design.rows.size();
    return 0;
}

int ref_netlist_export(void *hp, uint32_t *movVertex, uint32_t *varOfVertex, double *fixedX,
                       double *fixedY, uint64_t *netStart, uint32_t *pinCell, double *offX,
                       double *offY, double *netWeight, uint64_t *pinStart, uint32_t *pinNet,
                       uint32_t *pinQ, double *width, double *height, double *die4,
                       double *obstacles, double *rows) {
    auto *h = static_cast<Handle *>(hp);
    const Design &d = h->design;
    const Netlist &nl = d.netlist;
    std::copy(nl.movVertex.begin(), nl.movVertex.end(), movVertex);
    std::copy(nl.varOfVertex.begin(), nl.varOfVertex.end(), varOfVertex);
    std::copy(nl.fixedX.begin(), nl.fixedX.end(), fixedX);
    std::copy(nl.fixedY.begin(), nl.fixedY.end(), fixedY);
    uint64_t p = 0;
    netStart[0] = 0;
    for (std::size_t n = 0; n < nl.nets.size(); ++n) {
        const NetPins &np = nl.nets[n];
        for (std::size_t q = 0; q < np.cells.size(); ++q, ++p) {
            pinCell[p] = np.cells[q];
            offX[p] = np.offX[q];
            offY[p] = np.offY[q];
        }
        netStart[n + 1] = p;
        netWeight[n] = np.weight;
    }
    for (std::size_t i = 0; i < nl.pinStart.size(); ++i) pinStart[i] = nl.pinStart[i];
    for (std::size_t e = 0; e < nl.pinsOfCell.size(); ++e) {
        pinNet[e] = nl.pinsOfCell[e].net;
        pinQ[e] = nl.pinsOfCell[e].pin;
    }
    std::copy(d.width.begin(), d.width.end(), width);
    std::copy(d.height.begin(), d.height.end(), height);
    die4[0] = d.die.lowerLeft.x;
    die4[1] = d.die.lowerLeft.y;
    die4[2] = d.die.upperRight.x;
    die4[3] = d.die.upperRight.y;
    for (std::size_t o = 0; o < d.obstacles.size(); ++o) {
        obstacles[4 * o] = d.obstacles[o].lowerLeft.x;
        obstacles[4 * o + 1] = d.obstacles[o].lowerLeft.y;
        obstacles[4 * o + 2] = d.obstacles[o].upperRight.x;
        obstacles[4 * o + 3] = d.obstacles[o].upperRight.y;
    }
    for (std::size_t r = 0; r < d.rows.size(); ++r) {
        const simpl::RowInfo &ri = d.rows[r];
        rows[5 * r] = ri.coordinate;
        rows[5 * r + 1] = ri.height;
        rows[5 * r + 2] = ri.getPitch();
        rows[5 * r + 3] = ri.subrows.empty() ? 0.0 : ri.subrows.front().x.start;
        rows[5 * r + 4] = ri.subrows.empty() ? 0.0 : ri.subrows.back().x.end;
    }
    return 0;
}

int ref_floors(void *hp, double *fx, double *fy) {
    auto *h = static_cast<Handle *>(hp);
    auto &im = h->impl();
    *fx = im.*reach(FloorXTag{});
    *fy = im.*reach(FloorYTag{});
    return 0;
}

// LinearSystems::buildB2B with the floors of Impl::collect (or the given ones
// when floorX > 0). Anchors may be null when alpha <= 0.
int ref_build_b2b(void *hp, const double *x, const double *y, double alpha, const double *ax,
                  const double *ay, double floorX, double floorY) {
    auto *h = static_cast<Handle *>(hp);
    return guarded(h, [&] {
        const std::size_t n = h->design.netlist.numMovable;
        std::vector<double> vx(x, x + n), vy(y, y + n), vax, vay;
        if (ax != nullptr) vax.assign(ax, ax + n);
        if (ay != nullptr) vay.assign(ay, ay + n);
        auto &im = h->impl();
        const double fx = floorX > 0.0 ? floorX : im.*reach(FloorXTag{});
        const double fy = floorY > 0.0 ? floorY : im.*reach(FloorYTag{});
        LinearSystems ls{.netlist = h->design.netlist, .sysX = h->sysX, .sysY = h->sysY,
                         .floorX = fx, .floorY = fy};
        ls.buildB2B(vx, vy, alpha, vax, vay);
    });
}

// LinearSystems::buildStar; returns the extended system size in *size.
int ref_build_star(void *hp, uint64_t *size) {
    auto *h = static_cast<Handle *>(hp);
    return guarded(h, [&] {
        auto &im = h->impl();
        LinearSystems ls{.netlist = h->design.netlist, .sysX = h->sysX, .sysY = h->sysY,
                         .floorX = im.*reach(FloorXTag{}), .floorY = im.*reach(FloorYTag{})};
        *size = ls.buildStar();
    });
}

int ref_system_sizes(void *hp, int axis, uint64_t *n, uint64_t *m) {
    auto *h = static_cast<Handle *>(hp);
    const SparseSystem &s = axis == 0 ? h->sysX : h->sysY;
    *n = s.size();
    *m = s.rowPtr.empty() ? 0 : s.rowPtr.back();
    return 0;
}

int ref_system_export(void *hp, int axis, uint64_t *rowPtr, uint32_t *col, double *val,
                      double *diag, double *rhs) {
    auto *h = static_cast<Handle *>(hp);
    const SparseSystem &s = axis == 0 ? h->sysX : h->sysY;
    for (std::size_t i = 0; i < s.rowPtr.size(); ++i) rowPtr[i] = s.rowPtr[i];
    std::copy(s.col.begin(), s.col.end(), col);
    std::copy(s.val.begin(), s.val.end(), val);
    std::copy(s.diag.begin(), s.diag.end(), diag);
    std::copy(s.rhs.begin(), s.rhs.end(), rhs);
    return 0;
}

// Replaces the stored system of one axis (used to solve systems that were
// produced elsewhere, e.g. by the GPU build, with the reference solver).
int ref_system_import(void *hp, int axis, uint64_t n, const uint64_t *rowPtr, const uint32_t *col,
                      const double *val, const double *diag, const double *rhs) {
    auto *h = static_cast<Handle *>(hp);
    SparseSystem &s = axis == 0 ? h->sysX : h->sysY;
    s.rowPtr.assign(rowPtr, rowPtr + n + 1);
    s.col.assign(col, col + rowPtr[n]);
    s.val.assign(val, val + rowPtr[n]);
    s.diag.assign(diag, diag + n);
    s.rhs.assign(rhs, rhs + n);
    return 0;
}

// solveBothAxes on the stored systems. x, y are updated in place. The
// observer records the per-iterate residuals (histCap entries per axis).
int ref_solve(void *hp, double *x, double *y, double tol, uint64_t maxIter, double *resid2,
              double *histX, double *histY, uint64_t histCap, uint64_t *iters) {
    auto *h = static_cast<Handle *>(hp);
    return guarded(h, [&] {
        std::vector<double> vx(x, x + h->sysX.size()), vy(y, y + h->sysY.size());
        uint64_t count = 0;
        const IterateObserver observe = [&](std::size_t it, const Residuals &r, bool) {
            if (it - 1 < histCap) {
                if (histX) histX[it - 1] = r.x;
                if (histY) histY[it - 1] = r.y;
            }
            count = it;
        };
        const Residuals r = solveBothAxes(h->sysX, vx, h->sysY, vy, tol, maxIter, observe);
        std::copy(vx.begin(), vx.end(), x);
        std::copy(vy.begin(), vy.end(), y);
        resid2[0] = r.x;
        resid2[1] = r.y;
        if (iters) *iters = count;
    });
}

double ref_hpwl(void *hp, const double *x, const double *y) {
    auto *h = static_cast<Handle *>(hp);
    const std::size_t n = h->design.netlist.numMovable;
    std::vector<double> vx(x, x + n), vy(y, y + n);
    auto &im = h->impl();
    return (im.*reach(HpwlTag{}))(vx, vy);
}

// Impl::buildGrid(perAxis); info = origin.x, origin.y, dx, dy, nx, ny,
// totalAvail. avail (nx*ny, row-major iy*nx+ix) may be null.
int ref_grid(void *hp, uint64_t perAxis, double densityLimit, double *info, double *avail) {
    auto *h = static_cast<Handle *>(hp);
    return guarded(h, [&] {
        auto &im = h->impl();
        (im.*reach(BuildGridTag{}))(perAxis);
        im.*reach(DensityTag{}) = std::clamp(densityLimit, 0.05, 1.0);
        const BinGrid &g = im.*reach(GridTag{});
        info[0] = g.origin.x;
        info[1] = g.origin.y;
        info[2] = g.dx;
        info[3] = g.dy;
        info[4] = static_cast<double>(g.nx);
        info[5] = static_cast<double>(g.ny);
        info[6] = g.totalAvail;
        if (avail) std::copy(g.avail.begin(), g.avail.end(), avail);
    });
}

// Full SimPL run (simplDM::run, simpl_dm.cc:245-248) on a copy of the design.
// opts: cgTol, cgMaxIter, maxIters, initMaxIters, seed, alphaBase,
// binsPerAxis, densityLimit, refineIters; initNet: "star" | "b2b" |
// "star_b2b". Final (look-ahead legalized) positions go to x, y.
int ref_run_simpl(void *hp, const double *opts, const char *initNet, double *x, double *y) {
    auto *h = static_cast<Handle *>(hp);
    return guarded(h, [&] {
        SimplOptions o;
        o.cgTol = opts[0];
        o.cgMaxIter = static_cast<std::size_t>(opts[1]);
        o.maxIters = static_cast<std::size_t>(opts[2]);
        o.initMaxIters = static_cast<std::size_t>(opts[3]);
        o.seed = static_cast<std::size_t>(opts[4]);
        o.alphaBase = opts[5];
        o.binsPerAxis = static_cast<std::size_t>(opts[6]);
        o.densityLimit = opts[7];
        o.refineIters = static_cast<std::size_t>(opts[8]);
        o.initialNetModel = initNet;
        o.fences = false;
        o.reportEvery = 0;
        o.traceEvery = 0;
        o.cgEvery = 0;
        o.initCgEvery = 0;
        simplDM dm(h->design, o);
        dm.run();
        const Design &d = dm.getDesign();
        std::copy(d.x.begin(), d.x.end(), x);
        std::copy(d.y.begin(), d.y.end(), y);
    });
}

// Impl::lookAheadLegalize on the grid of the last ref_grid (default
// SimplOptions: maxLevel 20, minCellsToSplit 4, stripeAreaFraction 0.1), in
// place on x, y.
int ref_lal(void *hp, double *x, double *y) {
    auto *h = static_cast<Handle *>(hp);
    return guarded(h, [&] {
        const std::size_t n = h->design.netlist.numMovable;
        std::vector<double> vx(x, x + n), vy(y, y + n);
        auto &im = h->impl();
        (im.*reach(LalTag{}))(vx, vy);
        std::copy(vx.begin(), vx.end(), x);
        std::copy(vy.begin(), vy.end(), y);
    });
}

// The FreeSpace rows of the last ref_grid: counts[0] = rows, counts[1] =
// spans; rows [R*2] (y start, y end), row_span [R+1] offsets, spans [S*2].
// Pointers may be null to query the counts.
int ref_free_space(void *hp, uint64_t *counts, double *rows, uint64_t *row_span, double *spans) {
    auto *h = static_cast<Handle *>(hp);
    return guarded(h, [&] {
        const FreeSpace &fs = h->impl().*reach(FreeTag{});
        uint64_t s = 0;
        for (std::size_t r = 0; r < fs.rows.size(); ++r) {
            if (rows) {
                rows[2 * r] = fs.rows[r].y.start;
                rows[2 * r + 1] = fs.rows[r].y.end;
            }
            if (row_span) row_span[r] = s;
            for (const Interval &sp : fs.rows[r].spans) {
                if (spans) {
                    spans[2 * s] = sp.start;
                    spans[2 * s + 1] = sp.end;
                }
                ++s;
            }
        }
        if (row_span) row_span[fs.rows.size()] = s;
        counts[0] = fs.rows.size();
        counts[1] = s;
    });
}

// Impl::getOccupancy then Impl::getOverflow on the grid of the last ref_grid.
int ref_occupancy(void *hp, const double *x, const double *y, double *occ, double *overflow) {
    auto *h = static_cast<Handle *>(hp);
    return guarded(h, [&] {
        const std::size_t n = h->design.netlist.numMovable;
        std::vector<double> vx(x, x + n), vy(y, y + n);
        auto &im = h->impl();
        const std::vector<double> o = (im.*reach(OccTag{}))(vx, vy);
        if (occ) std::copy(o.begin(), o.end(), occ);
        *overflow = (im.*reach(OverflowTag{}))(o);
    });
}

}  // extern "C"
