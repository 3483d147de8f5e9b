// Oracle harness around the reference's own Kraftwerk2 system build and CG
// (test infrastructure only).
//
// Compiled against the reference sources where they lie (oracle/Makefile)
// into oracle/_ref/libktref.so. Every number it returns is computed by
// reference code:
//   * kw2_build -> Kraftwerk2Placer::Impl::buildSystem
//                  (globalPlacer/kraftwerk2/kraftwerk2_placer.cc:328-410),
//                  after Impl::indexPins (kraftwerk2_placer.cc:302-326)
//   * kw2_solve -> solve (kraftwerk2_placer.cc:86-126)
// The Impl members are private to kraftwerk2_placer.cc, so that file is
// included here and its members are reached through the explicit-
// instantiation access rule ([temp.spec.general]); System and solve live in
// that file's unnamed namespace, which this translation unit shares.
//
// The Design is filled directly from the caller's arrays: the movable cells
// (slots) with width and height, and per net its pins as (slot or -1, offset,
// fixedPosition), exactly the fields kraftwerk2_dm.cc:34-54 sets.

#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "globalPlacer/kraftwerk2/kraftwerk2_placer.cc"

namespace {

using namespace ktplace;
using namespace ktplace::kraftwerk2;

template <typename Tag, auto Member>
struct Grant {
    friend auto reach(Tag) { return Member; }
};

struct KPImplTag { friend auto reach(KPImplTag); };
struct KBuildTag { friend auto reach(KBuildTag); };
struct KIndexTag { friend auto reach(KIndexTag); };
struct KFloorXTag { friend auto reach(KFloorXTag); };
struct KFloorYTag { friend auto reach(KFloorYTag); };

template <typename T>
struct MemberOf;
template <typename C, typename M>
struct MemberOf<M C::*> {
    using type = M;
};

}  // namespace

template struct Grant<KPImplTag, &Kraftwerk2Placer::pImpl>;
template struct Grant<KBuildTag, &Kraftwerk2Placer::Impl::buildSystem>;
template struct Grant<KIndexTag, &Kraftwerk2Placer::Impl::indexPins>;
template struct Grant<KFloorXTag, &Kraftwerk2Placer::Impl::floorX>;
template struct Grant<KFloorYTag, &Kraftwerk2Placer::Impl::floorY>;

namespace {

using ImplT = MemberOf<decltype(reach(KPImplTag{}))>::type::element_type;

struct KHandle {
    Design design;
    std::unique_ptr<ImplT> impl;
    System sys;
    std::string error;
};

}  // namespace

extern "C" {

void *kw2_create(int64_t n, const double *width, const double *height, int64_t num_nets,
                 const int64_t *net_start, const int64_t *pin_slot, const double *off_x,
                 const double *off_y, const double *fix_x, const double *fix_y,
                 const double *weight, double die_lx, double die_ly, double die_ux,
                 double die_uy) {
    try {
        auto h = std::make_unique<KHandle>();
        Design &d = h->design;
        for (int64_t i = 0; i < n; ++i) {
            d.cells.id.push_back(static_cast<std::size_t>(i));
            d.cells.x.push_back(0.0);
            d.cells.y.push_back(0.0);
            d.cells.width.push_back(width[i]);
            d.cells.height.push_back(height[i]);
        }
        std::vector<NetPin> pins;
        for (int64_t k = 0; k < num_nets; ++k) {
            pins.clear();
            for (int64_t p = net_start[k]; p < net_start[k + 1]; ++p) {
                pins.push_back(NetPin{.slot = pin_slot[p] < 0 ? noSlot
                                                              : static_cast<std::size_t>(pin_slot[p]),
                                      .offset = Point(off_x[p], off_y[p]),
                                      .fixedPosition = Point(fix_x[p], fix_y[p])});
            }
            d.nets.add(pins);
            d.netWeight.push_back(weight[k]);
        }
        d.die = BBox(Point(die_lx, die_ly), Point(die_ux, die_uy));
        h->impl = std::make_unique<ImplT>(d);
        ((*h->impl).*reach(KIndexTag{}))();
        return h.release();
    } catch (const std::exception &) {
        return nullptr;
    }
}

void kw2_destroy(void *p) { delete static_cast<KHandle *>(p); }

// buildSystem(horizontal, withRhs) at positions (x, y) with the given floors;
// returns the number of stored entries.
int64_t kw2_build(void *p, const double *x, const double *y, int horizontal, int with_rhs,
                  double floor_x, double floor_y) {
    auto *h = static_cast<KHandle *>(p);
    Design &d = h->design;
    std::memcpy(d.cells.x.data(), x, sizeof(double) * d.cells.size());
    std::memcpy(d.cells.y.data(), y, sizeof(double) * d.cells.size());
    (*h->impl).*reach(KFloorXTag{}) = floor_x;
    (*h->impl).*reach(KFloorYTag{}) = floor_y;
    h->sys = System{};
    ((*h->impl).*reach(KBuildTag{}))(horizontal != 0, with_rhs != 0, h->sys);
    return static_cast<int64_t>(h->sys.col.size());
}

void kw2_get_system(void *p, int64_t *row_start, int32_t *col, double *val, double *diag,
                    double *rhs) {
    const System &s = static_cast<KHandle *>(p)->sys;
    for (std::size_t i = 0; i < s.rowStart.size(); ++i) row_start[i] = static_cast<int64_t>(s.rowStart[i]);
    for (std::size_t e = 0; e < s.col.size(); ++e) {
        col[e] = static_cast<int32_t>(s.col[e]);
        val[e] = s.val[e];
    }
    std::memcpy(diag, s.diag.data(), sizeof(double) * s.diag.size());
    std::memcpy(rhs, s.rhs.data(), sizeof(double) * s.rhs.size());
}

// Replaces the kept system's diag and rhs (the caller's adjustments).
void kw2_set_diag_rhs(void *p, const double *diag, const double *rhs) {
    System &s = static_cast<KHandle *>(p)->sys;
    std::memcpy(s.diag.data(), diag, sizeof(double) * s.diag.size());
    std::memcpy(s.rhs.data(), rhs, sizeof(double) * s.rhs.size());
}

// The reference's solve on the kept system, in place on x.
void kw2_solve(void *p, double *x, double tol, int64_t max_iter) {
    auto *h = static_cast<KHandle *>(p);
    std::vector<double> v(x, x + h->sys.diag.size());
    solve(h->sys, v, tol, static_cast<std::size_t>(max_iter));
    std::memcpy(x, v.data(), sizeof(double) * v.size());
}

}  // extern "C"
