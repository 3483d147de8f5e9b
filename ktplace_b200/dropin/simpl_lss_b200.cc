// Drop-in replacement for KTPlace's globalPlacer/simpl/simpl_lss.cc.
//
// Compiled against the reference's own header (globalPlacer/simpl/
// simpl_lss.h), it defines the same three symbols the SimPL placer calls and
// runs them on a B200 through the ktplace_b200 C ABI:
//
//   LinearSystems::buildB2B  (reference: simpl_lss.cc:11-114)  -> ktg_build_b2b
//   LinearSystems::buildStar (reference: simpl_lss.cc:116-201) -> ktg_build_star
//   solveBothAxes            (reference: simpl_lss.cc:203-290) -> ktg_solve
//
// Link this object instead of simpl_lss.o. One GPU
// context per process (device $KTPLACE_B200_DEVICE, default 0) holds the
// netlist, uploaded the first time a Netlist is seen and again whenever a
// different one is. Errors from the GPU are fatal through ktlog, as the
// reference treats its own unrecoverable states.
//
// Contract differences from the reference's simpl_lss.cc:
//   * with $KTPLACE_B200_HOST_CSR=0 buildB2B fills only diag and rhs on the
//     host and leaves rowPtr/col/val empty; solveBothAxes then uses the device
//     copy. By default the whole CSR is copied back, as the reference fills it.
//   * the IterateObserver is replayed after the device solve with each
//     iterate's residuals; x and y already hold the final solution then.
//   * solveBothAxes sums its dot products in the reference's order
//     (pcg_form 2), so solutions, iteration counts and residuals are the
//     reference's bit for bit; $KTPLACE_B200_PCG_FORM=3 selects the library's
//     default (faster) form, whose results agree to about 1e-9 relative.
#include "globalPlacer/simpl/simpl_lss.h"
#include "util/kt_log.h"

#include "ktplace_b200.h"
#include "simpl_hooks_b200.h"

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

namespace ktplace::simpl {
namespace {

struct GpuState {
    ktg_ctx *ctx = nullptr;
    const Netlist *netlist = nullptr;
    std::size_t netlistMovable = 0;
    std::size_t netlistNets = 0;
    // The SparseSystem objects whose device copy is current.
    const SparseSystem *devX = nullptr;
    const SparseSystem *devY = nullptr;
    std::size_t devRows = 0;
    bool hostCsr = true;
    std::vector<double> histX, histY;
    bool sizes = false;  // the uploaded netlist carries the cells' real sizes
    // the bin grid installed for ktg_occupancy
    std::size_t gridNx = 0, gridNy = 0;
    double gridOx = 0.0, gridOy = 0.0, gridDx = 0.0, gridDy = 0.0, gridTotal = -1.0;
    double gridLimit = -1.0;
};

GpuState &state() {
    static GpuState s;
    return s;
}

[[noreturn]] void fail(const char *what, int rc) {
    const ktg_ctx *c = state().ctx;
    ktlog.fatal("ktplace_b200: {} failed ({}): {}", what, rc, c ? ktg_last_error(c) : "");
}

void check(const char *what, int rc) {
    if (rc != KTG_OK) fail(what, rc);
}

ktg_ctx *context() {
    GpuState &s = state();
    if (s.ctx == nullptr) {
        const char *dev = std::getenv("KTPLACE_B200_DEVICE");
        const char *csr = std::getenv("KTPLACE_B200_HOST_CSR");
        const char *form = std::getenv("KTPLACE_B200_PCG_FORM");
        s.hostCsr = !(csr != nullptr && std::string(csr) == "0");
        check("ktg_create", ktg_create(dev ? std::atoi(dev) : 0, &s.ctx));
        check("ktg_set_option", ktg_set_option(s.ctx, "pcg_form", form ? std::atoi(form) : 2));
        const char *ho = std::getenv("KTPLACE_B200_HPWL_ORDER");
        check("ktg_set_option", ktg_set_option(s.ctx, "hpwl_order", ho ? std::atoi(ho) : 2));
    }
    return s.ctx;
}

// SimPL's Netlist as the C ABI's structure of arrays (one-time per design;
// again once when the density hook first brings the cells' sizes).
void ensureNetlist(const Netlist &nl, const std::vector<double> *width = nullptr,
                   const std::vector<double> *height = nullptr) {
    GpuState &s = state();
    ktg_ctx *c = context();
    if (s.netlist == &nl && s.netlistMovable == nl.numMovable && s.netlistNets == nl.nets.size() &&
        (width == nullptr || s.sizes))
        return;
    const std::size_t V = nl.varOfVertex.size();
    const std::size_t n = nl.numMovable;
    std::vector<int32_t> movVertex(nl.movVertex.begin(), nl.movVertex.end());
    std::vector<int32_t> varOf(V);
    for (std::size_t v = 0; v < V; ++v)
        varOf[v] = nl.varOfVertex[v] == noVar ? -1 : static_cast<int32_t>(nl.varOfVertex[v]);
    std::vector<int64_t> netStart(nl.nets.size() + 1, 0);
    for (std::size_t k = 0; k < nl.nets.size(); ++k)
        netStart[k + 1] = netStart[k] + static_cast<int64_t>(nl.nets[k].cells.size());
    std::vector<int32_t> pinCell(netStart.back());
    std::vector<double> offX(netStart.back()), offY(netStart.back()), weight(nl.nets.size());
    for (std::size_t k = 0; k < nl.nets.size(); ++k) {
        const NetPins &np = nl.nets[k];
        weight[k] = np.weight;
        for (std::size_t q = 0; q < np.cells.size(); ++q) {
            pinCell[netStart[k] + q] = static_cast<int32_t>(np.cells[q]);
            offX[netStart[k] + q] = np.offX[q];
            offY[netStart[k] + q] = np.offY[q];
        }
    }
    std::vector<int64_t> pinStart(nl.pinStart.begin(), nl.pinStart.end());
    std::vector<int32_t> pinNet(nl.pinsOfCell.size()), pinQ(nl.pinsOfCell.size());
    for (std::size_t e = 0; e < nl.pinsOfCell.size(); ++e) {
        pinNet[e] = static_cast<int32_t>(nl.pinsOfCell[e].net);
        pinQ[e] = static_cast<int32_t>(nl.pinsOfCell[e].pin);
    }
    // Cell sizes are not part of Netlist: the density hook hands over the
    // placer's (Design::width/height); until then unit sizes keep the upload
    // valid for the assembly and solve.
    std::vector<double> ones(std::max<std::size_t>(n, 1), 1.0);
    const double *w = width ? width->data() : ones.data();
    const double *h = height ? height->data() : ones.data();
    ktg_netlist_view view{static_cast<int64_t>(V), static_cast<int64_t>(n),
                          static_cast<int64_t>(nl.nets.size()), movVertex.data(), varOf.data(),
                          nl.fixedX.data(), nl.fixedY.data(), netStart.data(), pinCell.data(),
                          offX.data(), offY.data(), weight.data(), pinStart.data(), pinNet.data(),
                          pinQ.data(), w, h};
    check("ktg_upload_netlist", ktg_upload_netlist(c, &view));
    s.sizes = width != nullptr;
    s.gridNx = s.gridNy = 0;  // the grid goes with the old upload
    s.netlist = &nl;
    s.netlistMovable = n;
    s.netlistNets = nl.nets.size();
    s.devX = s.devY = nullptr;
}

void download(ktg_ctx *c, int axis, SparseSystem &sys, bool hostCsr) {
    int64_t n = 0, m = 0;
    check("ktg_system_info", ktg_system_info(c, axis, &n, &m));
    sys.diag.resize(n);
    sys.rhs.resize(n);
    if (hostCsr) {
        std::vector<int64_t> rp(n + 1);
        std::vector<int32_t> col(m);
        sys.val.resize(m);
        check("ktg_download_system", ktg_download_system(c, axis, rp.data(), col.data(),
                                                         sys.val.data(), sys.diag.data(),
                                                         sys.rhs.data()));
        sys.rowPtr.assign(rp.begin(), rp.end());
        sys.col.assign(col.begin(), col.end());
    } else {
        check("ktg_download_system", ktg_download_system(c, axis, nullptr, nullptr, nullptr,
                                                         sys.diag.data(), sys.rhs.data()));
        sys.rowPtr.clear();
        sys.col.clear();
        sys.val.clear();
    }
}

void upload(ktg_ctx *c, int axis, const SparseSystem &sys) {
    const std::size_t n = sys.size();
    if (sys.rowPtr.size() != n + 1)
        ktlog.fatal("ktplace_b200: system of axis {} has no CSR on the host", axis);
    std::vector<int64_t> rp(sys.rowPtr.begin(), sys.rowPtr.end());
    std::vector<int32_t> col(sys.col.begin(), sys.col.end());
    check("ktg_upload_system",
          ktg_upload_system(c, axis, static_cast<int64_t>(n), rp.data(), col.data(),
                            sys.val.data(), sys.diag.data(), sys.rhs.data()));
}

}  // namespace

void LinearSystems::buildB2B(const std::vector<double> &x, const std::vector<double> &y,
                             double alpha, const std::vector<double> &anchorX,
                             const std::vector<double> &anchorY) const {
    ensureNetlist(netlist);
    GpuState &s = state();
    ktg_ctx *c = s.ctx;
    check("ktg_set_pointer_mode", ktg_set_pointer_mode(c, KTG_PTR_HOST));
    const bool anchored = alpha > 0.0;
    check("ktg_build_b2b",
          ktg_build_b2b(c, x.data(), y.data(), alpha, anchored ? anchorX.data() : nullptr,
                        anchored ? anchorY.data() : nullptr, floorX, floorY));
    download(c, KTG_AXIS_X, sysX, s.hostCsr);
    download(c, KTG_AXIS_Y, sysY, s.hostCsr);
    s.devX = &sysX;
    s.devY = &sysY;
    s.devRows = sysX.size();
}

// Star model (simpl_lss.cc:116-201): assembled on the GPU by ktg_build_star
// (bit-identical to the reference) and copied into sysX/sysY like buildB2B.
std::size_t LinearSystems::buildStar() const {
    ensureNetlist(netlist);
    GpuState &s = state();
    ktg_ctx *c = s.ctx;
    int64_t size = 0;
    check("ktg_build_star", ktg_build_star(c, &size));
    download(c, KTG_AXIS_X, sysX, s.hostCsr);
    download(c, KTG_AXIS_Y, sysY, s.hostCsr);
    s.devX = &sysX;
    s.devY = &sysY;
    s.devRows = static_cast<std::size_t>(size);
    return static_cast<std::size_t>(size);
}

Residuals solveBothAxes(const SparseSystem &sysX, std::vector<double> &x, const SparseSystem &sysY,
                        std::vector<double> &y, double tolerance, std::size_t maxIterations,
                        const IterateObserver &observe) {
    GpuState &s = state();
    ktg_ctx *c = context();
    check("ktg_set_pointer_mode", ktg_set_pointer_mode(c, KTG_PTR_HOST));
    const bool current = s.devX == &sysX && s.devY == &sysY && s.devRows == sysX.size() &&
                         sysY.size() == sysX.size();
    if (!current) {
        upload(c, KTG_AXIS_X, sysX);
        upload(c, KTG_AXIS_Y, sysY);
        s.devX = &sysX;
        s.devY = &sysY;
        s.devRows = sysX.size();
    }
    const int64_t cap = observe ? static_cast<int64_t>(std::min<std::size_t>(maxIterations, 1u << 20)) : 0;
    s.histX.resize(cap);
    s.histY.resize(cap);
    ktg_solve_info info{};
    check("ktg_solve", ktg_solve(c, x.data(), y.data(), tolerance, static_cast<int64_t>(maxIterations),
                                 &info, cap ? s.histX.data() : nullptr,
                                 cap ? s.histY.data() : nullptr, cap));
    if (observe) {
        const std::size_t k = static_cast<std::size_t>(std::min<int64_t>(info.iters, cap));
        for (std::size_t it = 1; it <= k; ++it)
            observe(it, Residuals(s.histX[it - 1], s.histY[it - 1]), it == k && info.live == 0);
    }
    return Residuals(info.resid_x, info.resid_y);
}

namespace b200 {

double hpwl(const Netlist &netlist, const std::vector<double> &x, const std::vector<double> &y) {
    ensureNetlist(netlist);
    ktg_ctx *c = state().ctx;
    check("ktg_set_pointer_mode", ktg_set_pointer_mode(c, KTG_PTR_HOST));
    double h = 0.0;
    check("ktg_hpwl", ktg_hpwl(c, x.data(), y.data(), &h));
    return h;
}

std::vector<double> occupancy(const Netlist &netlist, const std::vector<double> &width,
                              const std::vector<double> &height, const BinGrid &grid,
                              double densityLimit, const std::vector<double> &x,
                              const std::vector<double> &y) {
    GpuState &s = state();
    ensureNetlist(netlist, &width, &height);
    ktg_ctx *c = s.ctx;
    if (s.gridNx != grid.nx || s.gridNy != grid.ny || s.gridOx != grid.origin.x ||
        s.gridOy != grid.origin.y || s.gridDx != grid.dx || s.gridDy != grid.dy ||
        s.gridTotal != grid.totalAvail || s.gridLimit != densityLimit) {
        const ktg_grid_view g{grid.origin.x, grid.origin.y, grid.dx, grid.dy,
                              static_cast<int64_t>(grid.nx), static_cast<int64_t>(grid.ny),
                              grid.avail.data(), grid.totalAvail, densityLimit};
        check("ktg_set_grid", ktg_set_grid(c, &g));
        s.gridNx = grid.nx;
        s.gridNy = grid.ny;
        s.gridOx = grid.origin.x;
        s.gridOy = grid.origin.y;
        s.gridDx = grid.dx;
        s.gridDy = grid.dy;
        s.gridTotal = grid.totalAvail;
        s.gridLimit = densityLimit;
    }
    check("ktg_set_pointer_mode", ktg_set_pointer_mode(c, KTG_PTR_HOST));
    std::vector<double> occ(grid.size(), 0.0);
    double overflow = 0.0;
    check("ktg_occupancy", ktg_occupancy(c, x.data(), y.data(), occ.data(), &overflow));
    return occ;
}

}  // namespace b200

}  // namespace ktplace::simpl
