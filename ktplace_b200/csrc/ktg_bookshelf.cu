// Bookshelf reader feeding ktg_upload_netlist (host code, multithreaded).
//
// Reads <dir>/<name>.nodes/.wts/.nets/.pl/.scl (name = the directory's own
// name; ".gz" variants through zlib, which also reads plain files) with the
// rules of the reference's BookshelfInputAdapter (adaptor/
// bookshelfToKTAdaptor.cc:137-672), then flattens the design the way
// buildSimplDM does (globalPlacer/simpl/simpl_dm.cc:16-85,262-279, datamodel/
// kt_die.cc:45-105), so the arrays match the reference's design bit for bit:
//   .nodes  the header ends at the first line holding "NumTerminals"; a body
//           line is "name width height [terminal]" (only the exact word
//           "terminal" fixes the cell); a repeated name keeps the first;
//   .wts    "net weight" lines (a later line overrides an earlier one);
//   .nets   "NetDegree [:] d [name]" opens a net, the following non-empty
//           lines are its pins; net k reads min(lines, d) of them from the
//           list of all pin lines at the sum of the earlier nets' minima (so
//           surplus lines shift later nets, as in the reference); a pin is
//           "cell dir [: dx dy]" (offset from the cell centre); a name-less
//           net is called "n<index>"; a repeated net name adds its pins to the
//           first net of that name (whose weight stays); pins of unknown cells
//           are dropped;
//   .pl     "name x y ..." sets the position, a "/FIXED" token fixes the cell;
//           a malformed coordinate aborts the read, as the reference's
//           uncaught std::stod does;
//   .scl    CoreRow ... End blocks, case-insensitive keys, several
//           SubrowOrigin/NumSites pairs per row; rows without sites dropped.
// Numbers go through strtod like std::stod, so they convert identically.
// Line parsing runs on `threads` host threads; everything that assigns ids
// (cells, nets, pins) runs in file order.
#include <zlib.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <limits>
#include <string>
#include <string_view>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ktplace_b200.h"

namespace {

thread_local std::string g_error;

struct Text {
    std::string data;
    std::vector<std::string_view> lines;
};

bool read_text(const std::string &path, Text &t) {
    const bool gz = path.size() > 3 && path.compare(path.size() - 3, 3, ".gz") == 0;
    if (!gz) {
        FILE *f = std::fopen(path.c_str(), "rb");
        if (!f) return false;
        std::fseek(f, 0, SEEK_END);
        const long size = std::ftell(f);
        std::fseek(f, 0, SEEK_SET);
        t.data.resize(size > 0 ? static_cast<size_t>(size) : 0);
        const size_t got = t.data.empty() ? 0 : std::fread(&t.data[0], 1, t.data.size(), f);
        std::fclose(f);
        if (got != t.data.size()) return false;
    } else {
        gzFile f = gzopen(path.c_str(), "rb");
        if (!f) return false;
        gzbuffer(f, 1 << 20);
        std::vector<char> buf(1 << 22);
        int got;
        while ((got = gzread(f, buf.data(), static_cast<unsigned>(buf.size()))) > 0)
            t.data.append(buf.data(), static_cast<size_t>(got));
        const bool ok = got == 0;
        gzclose(f);
        if (!ok) return false;
    }
    const char *b = t.data.data();
    const size_t n = t.data.size();
    t.lines.reserve(n / 24 + 16);
    size_t s = 0;
    while (s < n) {
        const void *nl = std::memchr(b + s, '\n', n - s);
        const size_t e = nl ? static_cast<size_t>(static_cast<const char *>(nl) - b) : n;
        t.lines.emplace_back(b + s, e - s);
        s = e + 1;
    }
    return true;
}

// Open-addressing map from names (views into file text that outlive it) to
// ids; hashes are computed up front (in parallel) and inserts keep the
// caller's order, so ids are assigned in file order.
class NameMap {
public:
    void reserve(size_t n) {
        size_t cap = 16;
        while (cap < 2 * n + 16) cap <<= 1;
        slots_.assign(cap, Slot{});
        mask_ = cap - 1;
    }
    static uint64_t hash(std::string_view s) {  // FNV-1a
        uint64_t h = 1469598103934665603ull;
        for (unsigned char c : s) {
            h ^= c;
            h *= 1099511628211ull;
        }
        return h;
    }
    // id of `s` if present, else inserts `id` and returns it
    int32_t find_or_insert(std::string_view s, uint64_t h, int32_t id) {
        for (size_t i = h & mask_;; i = (i + 1) & mask_) {
            Slot &sl = slots_[i];
            if (sl.id < 0) {
                sl = Slot{h, s, id};
                return id;
            }
            if (sl.h == h && sl.key == s) return sl.id;
        }
    }
    int32_t find(std::string_view s, uint64_t h) const {
        for (size_t i = h & mask_;; i = (i + 1) & mask_) {
            const Slot &sl = slots_[i];
            if (sl.id < 0) return -1;
            if (sl.h == h && sl.key == s) return sl.id;
        }
    }

private:
    struct Slot {
        uint64_t h = 0;
        std::string_view key;
        int32_t id = -1;
    };
    std::vector<Slot> slots_;
    size_t mask_ = 0;
};

// The file itself, or its ".gz" twin when that exists (the reference prefers it).
std::string pick(const std::string &base, const char *ext) {
    const std::string plain = base + ext;
    std::error_code ec;
    if (std::filesystem::exists(plain + ".gz", ec)) return plain + ".gz";
    return plain;
}

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; }
bool is_ws(char c) {  // what operator>> skips
    return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

std::string_view strip(std::string_view s) {
    const size_t hash = s.find('#');
    if (hash != std::string_view::npos) s = s.substr(0, hash);
    size_t a = 0, b = s.size();
    while (a < b && is_space(s[a])) ++a;
    while (b > a && is_space(s[b - 1])) --b;
    return s.substr(a, b - a);
}

void tokenize(std::string_view s, std::vector<std::string_view> &out) {
    out.clear();
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && is_ws(s[i])) ++i;
        size_t j = i;
        while (j < s.size() && !is_ws(s[j])) ++j;
        if (j > i) out.push_back(s.substr(i, j - i));
        i = j;
    }
}

// std::stod: the longest valid prefix; no conversion or a range error fails.
bool to_double(std::string_view tok, double &v) {
    char small[96];
    std::string big;
    const char *p;
    if (tok.size() < sizeof(small)) {
        std::memcpy(small, tok.data(), tok.size());
        small[tok.size()] = '\0';
        p = small;
    } else {
        big.assign(tok);
        p = big.c_str();
    }
    char *end = nullptr;
    errno = 0;
    const double d = std::strtod(p, &end);
    if (end == p || errno == ERANGE) return false;
    v = d;
    return true;
}

// std::stoull on a degree token (the reference lets the exception escape;
// such a file fails to read).
bool to_count(std::string_view tok, uint64_t &v) {
    std::string s(tok);
    char *end = nullptr;
    errno = 0;
    const unsigned long long d = std::strtoull(s.c_str(), &end, 10);
    if (end == s.c_str() || errno == ERANGE) return false;
    v = d;
    return true;
}

bool iequals(std::string_view a, const char *b) {
    if (a.size() != std::strlen(b)) return false;
    for (size_t i = 0; i < a.size(); ++i)
        if (std::tolower(static_cast<unsigned char>(a[i])) != std::tolower(static_cast<unsigned char>(b[i])))
            return false;
    return true;
}

template <typename F>
void parallel_for(int64_t n, int threads, F &&f) {
    if (threads <= 1 || n < 4096) {
        for (int64_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::vector<std::thread> pool;
    const int64_t per = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const int64_t a = t * per, b = std::min<int64_t>(n, a + per);
        if (a >= b) break;
        pool.emplace_back([&f, a, b] {
            for (int64_t i = a; i < b; ++i) f(i);
        });
    }
    for (auto &th : pool) th.join();
}

struct Cell {
    double width = 0.0, height = 0.0, x = 0.0, y = 0.0;
    bool terminal = false, fixed = false;
};

struct Pin {
    int32_t cell;
    double ox, oy;  // lower-left relative
};

struct Row {
    double coordinate, height, sitewidth, sitespacing;
    std::vector<std::pair<double, double>> subrows;  // (origin x, number of sites)
    double pitch() const { return sitespacing > 0.0 ? sitespacing : sitewidth; }
};

struct Raw {
    Text nodes_text;  // cell names point into it
    std::vector<Cell> cells;
    NameMap cell_id;
    std::vector<std::vector<Pin>> net_pins;
    std::vector<double> net_weight;
    std::vector<Row> rows;
};

bool parse_nodes(const std::string &path, int threads, Raw &r) {
    Text &t = r.nodes_text;
    if (!read_text(path, t)) {
        g_error = "cannot open the nodes file: " + path;
        return false;
    }
    size_t body = 0;
    while (body < t.lines.size()) {
        const bool found = strip(t.lines[body]).find("NumTerminals") != std::string_view::npos;
        ++body;
        if (found) break;
    }
    const int64_t count = static_cast<int64_t>(t.lines.size() - body);
    struct Rec {
        std::string_view name;
        uint64_t h = 0;
        double w = 0, h2 = 0;
        bool terminal = false, valid = false;
    };
    std::vector<Rec> recs(static_cast<size_t>(std::max<int64_t>(count, 0)));
    parallel_for(count, threads, [&](int64_t i) {
        thread_local std::vector<std::string_view> tok;
        const std::string_view s = strip(t.lines[body + i]);
        if (s.empty()) return;
        tokenize(s, tok);
        if (tok.size() < 3) return;
        Rec &rec = recs[i];
        if (!to_double(tok[1], rec.w) || !to_double(tok[2], rec.h2)) return;
        rec.terminal = tok.size() >= 4 && tok[3] == "terminal";
        rec.name = tok[0];
        rec.h = NameMap::hash(tok[0]);
        rec.valid = true;
    });
    r.cells.reserve(recs.size());
    r.cell_id.reserve(recs.size());
    for (const Rec &rec : recs) {
        if (!rec.valid) continue;
        const int32_t id = static_cast<int32_t>(r.cells.size());
        if (r.cell_id.find_or_insert(rec.name, rec.h, id) != id) continue;  // repeated name
        Cell c;
        c.width = rec.w;
        c.height = rec.h2;
        c.terminal = rec.terminal;
        c.fixed = rec.terminal;
        r.cells.push_back(c);
    }
    return true;
}

void parse_wts(const std::string &path, std::unordered_map<std::string, double> &w) {
    Text t;
    if (!read_text(path, t)) return;  // optional
    bool header = true;
    std::vector<std::string_view> tok;
    for (std::string_view line : t.lines) {
        const std::string_view s = strip(line);
        if (s.empty()) continue;
        if (header) {
            if (s.find("UCLA") != std::string_view::npos) continue;
            header = false;
        }
        tokenize(s, tok);
        if (tok.size() < 2) continue;
        double v;
        if (!to_double(tok[1], v)) continue;
        w[std::string(tok[0])] = v;
    }
}

bool starts_with_exactly(std::string_view s, size_t len, const char *word) {
    // std::string::compare(0, len, word) == 0
    return s.substr(0, len) == std::string_view(word);
}

bool parse_nets(const std::string &path, int threads, const std::unordered_map<std::string, double> &wts,
                Raw &r) {
    Text t;
    if (!read_text(path, t)) {
        g_error = "cannot open the nets file: " + path;
        return false;
    }
    const int64_t L = static_cast<int64_t>(t.lines.size());
    std::vector<std::string_view> stripped(t.lines.size());
    parallel_for(L, threads, [&](int64_t i) { stripped[i] = strip(t.lines[i]); });
    struct Stub {
        std::string_view name;
        uint64_t degree;
        uint64_t lines;  // pin lines seen after this header
    };
    std::vector<Stub> stubs;
    std::vector<int64_t> pin_lines;  // every pin line, in file order
    bool header = true;
    std::vector<std::string_view> tok;
    for (int64_t i = 0; i < L; ++i) {
        const std::string_view s = stripped[i];
        if (s.empty()) continue;
        if (header) {
            if (starts_with_exactly(s, 5, "UCLA") || starts_with_exactly(s, 7, "NumNets") ||
                starts_with_exactly(s, 7, "NumPins"))
                continue;
            header = false;
        }
        if (starts_with_exactly(s, 9, "NetDegree")) {
            tokenize(s, tok);
            size_t k = 1;
            while (k < tok.size() && tok[k] == ":") ++k;
            if (tok.size() < k + 1) continue;  // malformed header: skipped
            Stub st{std::string_view(), 0, 0};
            if (!to_count(tok[k], st.degree)) {
                g_error = "malformed net degree in " + path;
                return false;
            }
            st.name = k + 1 < tok.size() ? tok[k + 1] : std::string_view();
            stubs.push_back(std::move(st));
            continue;
        }
        if (!stubs.empty()) {
            pin_lines.push_back(i);
            ++stubs.back().lines;
        }
    }
    // Net k reads min(lines, degree) pin lines starting at the prefix sum of
    // those minima over the earlier nets, in the list of all pin lines: a net
    // with more lines than its degree shifts the pins of the nets after it, as
    // in the reference (bookshelfToKTAdaptor.cc:336-374).
    std::vector<uint64_t> first(stubs.size());
    uint64_t run = 0;
    for (size_t k = 0; k < stubs.size(); ++k) {
        first[k] = run;
        run += std::min(stubs[k].lines, stubs[k].degree);
    }
    // Pins: parsed, resolved to cells and converted to lower-left offsets in
    // parallel (the cell map is read-only here); an unknown cell is dropped.
    std::vector<std::vector<Pin>> pins(stubs.size());
    parallel_for(static_cast<int64_t>(stubs.size()), threads, [&](int64_t k) {
        thread_local std::vector<std::string_view> tk;
        const Stub &st = stubs[k];
        const size_t cnt = static_cast<size_t>(std::min<uint64_t>(st.lines, st.degree));
        std::vector<Pin> &out = pins[k];
        out.reserve(cnt);
        for (size_t p = 0; p < cnt; ++p) {
            tokenize(stripped[pin_lines[first[k] + p]], tk);
            if (tk.size() < 2) continue;
            double ox = 0.0, oy = 0.0;
            if (tk.size() >= 5 && tk[2] == ":") {
                if (!to_double(tk[3], ox) || !to_double(tk[4], oy)) continue;
            }
            const int32_t c = r.cell_id.find(tk[0], NameMap::hash(tk[0]));
            if (c < 0) continue;
            const Cell &cell = r.cells[c];
            out.push_back(Pin{c, ox + 0.5 * cell.width, oy + 0.5 * cell.height});
        }
    });
    // Net ids in file order; a repeated name adds to the first net of that name.
    // Name-less nets are called "n<index>" (kept alive in `generated`).
    std::vector<std::string> generated;
    for (size_t k = 0; k < stubs.size(); ++k)
        if (stubs[k].name.empty()) generated.push_back("n" + std::to_string(k));
    std::vector<std::string_view> names(stubs.size());
    std::vector<uint64_t> hashes(stubs.size());
    {
        size_t g = 0;
        for (size_t k = 0; k < stubs.size(); ++k)
            names[k] = stubs[k].name.empty() ? std::string_view(generated[g++]) : stubs[k].name;
    }
    parallel_for(static_cast<int64_t>(stubs.size()), threads,
                 [&](int64_t k) { hashes[k] = NameMap::hash(names[k]); });
    NameMap net_id;
    net_id.reserve(stubs.size());
    std::vector<int32_t> id_of(stubs.size());
    for (size_t k = 0; k < stubs.size(); ++k) {
        const int32_t fresh = static_cast<int32_t>(r.net_weight.size());
        const int32_t id = net_id.find_or_insert(names[k], hashes[k], fresh);
        if (id == fresh) {
            // the weight is looked up by the name as written ("" for a name-less net)
            const auto w = wts.find(std::string(stubs[k].name));
            r.net_weight.push_back(w != wts.end() ? w->second : 1.0);
        }
        id_of[k] = id;
    }
    r.net_pins.resize(r.net_weight.size());
    for (size_t k = 0; k < stubs.size(); ++k) {
        std::vector<Pin> &dst = r.net_pins[id_of[k]];
        if (dst.empty()) dst.swap(pins[k]);
        else dst.insert(dst.end(), pins[k].begin(), pins[k].end());
    }
    return true;
}

bool parse_pl(const std::string &path, int threads, Raw &r) {
    Text t;
    if (!read_text(path, t)) return true;  // optional
    const int64_t L = static_cast<int64_t>(t.lines.size());
    // header: leading lines holding "UCLA" (before the first other non-empty line)
    int64_t body = 0;
    while (body < L) {
        const std::string_view s = strip(t.lines[body]);
        if (!s.empty() && s.find("UCLA") == std::string_view::npos) break;
        ++body;
    }
    struct Rec {
        int32_t cell = -1;
        double x = 0, y = 0;
        bool fixed = false;
        int state = 0;  // 0 skip, 1 apply, 2 malformed coordinate
    };
    std::vector<Rec> recs(static_cast<size_t>(L - body));
    parallel_for(L - body, threads, [&](int64_t i) {
        thread_local std::vector<std::string_view> tok;
        const std::string_view s = strip(t.lines[body + i]);
        if (s.empty()) return;
        tokenize(s, tok);
        if (tok.size() < 3) return;
        Rec &rec = recs[i];
        if (!to_double(tok[1], rec.x) || !to_double(tok[2], rec.y)) {
            rec.state = 2;
            return;
        }
        for (std::string_view tk : tok)
            if (tk == "/FIXED") rec.fixed = true;
        const int32_t c = r.cell_id.find(tok[0], NameMap::hash(tok[0]));
        if (c < 0) return;
        rec.cell = c;
        rec.state = 1;
    });
    for (const Rec &rec : recs) {  // in file order: a later line wins
        if (rec.state == 2) {
            g_error = "malformed placement line in " + path;
            return false;
        }
        if (rec.state != 1) continue;
        Cell &c = r.cells[rec.cell];
        c.x = rec.x;
        c.y = rec.y;
        if (rec.fixed) c.fixed = true;
    }
    return true;
}

void parse_scl_row(const std::vector<std::string_view> &fields, Raw &r) {
    Row row{0.0, 0.0, 1.0, 1.0, {}};
    double origin = 0.0, sites = 0.0;
    bool have_origin = false;
    std::vector<std::string_view> parts;
    for (std::string_view f : fields) {
        tokenize(f, parts);
        if (parts.size() < 2) continue;
        size_t v = 1;
        while (v < parts.size() && parts[v] == ":") ++v;
        if (v >= parts.size()) continue;
        const std::string_view k = parts[0];
        double val;
        if (iequals(k, "coordinate")) {
            if (to_double(parts[v], val)) row.coordinate = val;
        } else if (iequals(k, "height")) {
            if (to_double(parts[v], val)) row.height = val;
        } else if (iequals(k, "sitewidth")) {
            if (to_double(parts[v], val)) row.sitewidth = val;
        } else if (iequals(k, "sitespacing")) {
            if (to_double(parts[v], val)) row.sitespacing = val;
        } else if (iequals(k, "subroworigin")) {
            // the previous subrow is closed before the new origin is read, as in
            // the reference (a malformed origin then leaves the rest untouched)
            if (have_origin && sites > 0.0) row.subrows.emplace_back(origin, sites);
            if (!to_double(parts[v], val)) continue;
            origin = val;
            have_origin = true;
            sites = 0.0;
            for (size_t p = 0; p + 1 < parts.size(); ++p) {
                if (iequals(parts[p], "numsites")) {
                    size_t m = p + 1;
                    while (m < parts.size() && parts[m] == ":") ++m;
                    double ns;
                    if (m < parts.size() && to_double(parts[m], ns)) sites = ns;
                    break;
                }
            }
        }
    }
    if (have_origin && sites > 0.0) row.subrows.emplace_back(origin, sites);
    if (!row.subrows.empty()) r.rows.push_back(std::move(row));
}

void parse_scl(const std::string &path, Raw &r) {
    Text t;
    if (!read_text(path, t)) return;  // optional
    std::vector<std::string_view> fields;
    bool in_row = false;
    for (std::string_view line : t.lines) {
        const std::string_view s = strip(line);
        if (s.empty()) continue;
        if (s.find("CoreRow") != std::string_view::npos) {
            in_row = true;
            fields.clear();
            continue;
        }
        if (s == "End") {
            if (in_row) {
                parse_scl_row(fields, r);
                in_row = false;
            }
            continue;
        }
        if (in_row) fields.push_back(s);
    }
}

}  // namespace

struct ktg_bookshelf {
    int64_t V = 0, n = 0, N = 0, P = 0, Pm = 0, num_fixed = 0;
    std::vector<int32_t> mov_vertex, var_of_vertex, pin_cell, pin_net, pin_q;
    std::vector<double> fixed_x, fixed_y, off_x, off_y, net_weight, width, height;
    std::vector<int64_t> net_start, pin_start;
    std::vector<double> obstacles;  // [K * 4]
    std::vector<double> rows;       // [R * 5] coordinate, height, pitch, first xlo, last xhi
    std::vector<double> subrows;    // [S * 3] row index, xlo, xhi
    double die[4] = {0, 0, 0, 0};
    double ms[6] = {0, 0, 0, 0, 0, 0};  // nodes, wts, nets, pl, scl, flatten
};

namespace {

// buildSimplDM: collectCells, collectNets, copyRows, getPlacementDieBox.
void flatten(const Raw &r, ktg_bookshelf &b) {
    const int64_t V = static_cast<int64_t>(r.cells.size());
    b.V = V;
    b.var_of_vertex.assign(V, -1);
    b.fixed_x.resize(V);
    b.fixed_y.resize(V);
    for (int64_t v = 0; v < V; ++v) {
        const Cell &c = r.cells[v];
        b.fixed_x[v] = c.x;
        b.fixed_y[v] = c.y;
        if (c.fixed || c.terminal) {
            if (c.width > 0.0 && c.height > 0.0) {
                b.obstacles.insert(b.obstacles.end(), {c.x, c.y, c.x + c.width, c.y + c.height});
            }
            ++b.num_fixed;
            continue;
        }
        b.var_of_vertex[v] = static_cast<int32_t>(b.n++);
        b.mov_vertex.push_back(static_cast<int32_t>(v));
        b.width.push_back(c.width);
        b.height.push_back(c.height);
    }
    const int64_t N = static_cast<int64_t>(r.net_pins.size());
    b.N = N;
    b.net_start.assign(N + 1, 0);
    b.net_weight = r.net_weight;
    std::vector<size_t> order;
    for (int64_t k = 0; k < N; ++k) {
        const std::vector<Pin> &pins = r.net_pins[k];
        order.resize(pins.size());
        for (size_t q = 0; q < pins.size(); ++q) order[q] = q;
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t a, size_t c) { return pins[a].cell < pins[c].cell; });
        int32_t last = -1;
        for (size_t q : order) {
            if (last >= 0 && pins[q].cell == last) continue;
            last = pins[q].cell;
            b.pin_cell.push_back(pins[q].cell);
            b.off_x.push_back(pins[q].ox);
            b.off_y.push_back(pins[q].oy);
        }
        b.net_start[k + 1] = static_cast<int64_t>(b.pin_cell.size());
    }
    b.P = static_cast<int64_t>(b.pin_cell.size());
    b.pin_start.assign(b.n + 1, 0);
    for (int64_t p = 0; p < b.P; ++p) {
        const int32_t v = b.var_of_vertex[b.pin_cell[p]];
        if (v >= 0) ++b.pin_start[v + 1];
    }
    for (int64_t i = 0; i < b.n; ++i) b.pin_start[i + 1] += b.pin_start[i];
    b.Pm = b.pin_start[b.n];
    b.pin_net.resize(b.Pm);
    b.pin_q.resize(b.Pm);
    std::vector<int64_t> cursor(b.pin_start.begin(), b.pin_start.end() - 1);
    for (int64_t k = 0; k < N; ++k) {
        for (int64_t p = b.net_start[k]; p < b.net_start[k + 1]; ++p) {
            const int32_t v = b.var_of_vertex[b.pin_cell[p]];
            if (v < 0) continue;
            b.pin_net[cursor[v]] = static_cast<int32_t>(k);
            b.pin_q[cursor[v]] = static_cast<int32_t>(p - b.net_start[k]);
            ++cursor[v];
        }
    }
    for (size_t ri = 0; ri < r.rows.size(); ++ri) {
        const Row &row = r.rows[ri];
        const double pitch = row.pitch();
        const double xlo = row.subrows.front().first;
        const double xhi = row.subrows.back().first + row.subrows.back().second * pitch;
        b.rows.insert(b.rows.end(), {row.coordinate, row.height, pitch, xlo, xhi});
        for (const auto &sr : row.subrows)
            b.subrows.insert(b.subrows.end(),
                             {static_cast<double>(ri), sr.first, sr.first + sr.second * pitch});
    }
    // getPlacementDieBox (a Bookshelf design declares no die area)
    const double inf = std::numeric_limits<double>::max();
    double lx = inf, ly = inf, ux = -inf, uy = -inf;
    for (const Cell &c : r.cells) {
        if (!c.fixed && !c.terminal) continue;
        lx = std::min(lx, c.x);
        ly = std::min(ly, c.y);
        ux = std::max(ux, c.x + std::max(c.width, 1.0));
        uy = std::max(uy, c.y + std::max(c.height, 1.0));
    }
    const bool have_fixed = ux > lx && uy > ly;
    double rlx = inf, rly = inf, rux = -inf, ruy = -inf;
    bool any_row = false;
    for (const Row &row : r.rows) {
        const double pitch = row.pitch();
        if (!(pitch > 0.0)) continue;
        double xhi = 0.0;
        for (const auto &sr : row.subrows) xhi = std::max(xhi, sr.first + sr.second * pitch);
        rlx = std::min(rlx, row.subrows.front().first);
        rly = std::min(rly, row.coordinate);
        rux = std::max(rux, xhi);
        ruy = std::max(ruy, row.coordinate + row.height);
        any_row = true;
    }
    if (any_row && rux > rlx && ruy > rly) {
        if (!have_fixed) {
            lx = rlx;
            ly = rly;
            ux = rux;
            uy = ruy;
        } else {
            lx = std::min(lx, rlx);
            ly = std::min(ly, rly);
            ux = std::max(ux, rux);
            uy = std::max(uy, ruy);
        }
    }
    b.die[0] = lx;
    b.die[1] = ly;
    b.die[2] = ux;
    b.die[3] = uy;
}

}  // namespace

extern "C" {

const char *ktg_bookshelf_last_error(void) { return g_error.c_str(); }

int ktg_bookshelf_read(const char *dir, int threads, ktg_bookshelf **out) {
    if (!dir || !out) return KTG_ERR_ARG;
    *out = nullptr;
    g_error.clear();
    try {
        if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
        const std::string d(dir);
        const std::string name = std::filesystem::path(d).filename().string();
        const std::string base = d + "/" + name;
        Raw raw;
        double ms[6];
        auto t = std::chrono::steady_clock::now();
        auto lap = [&t](double &slot) {
            const auto now = std::chrono::steady_clock::now();
            slot = std::chrono::duration<double, std::milli>(now - t).count();
            t = now;
        };
        if (!parse_nodes(pick(base, ".nodes"), threads, raw)) return KTG_ERR_ARG;
        lap(ms[0]);
        std::unordered_map<std::string, double> wts;
        parse_wts(pick(base, ".wts"), wts);
        lap(ms[1]);
        if (!parse_nets(pick(base, ".nets"), threads, wts, raw)) return KTG_ERR_ARG;
        lap(ms[2]);
        if (!parse_pl(pick(base, ".pl"), threads, raw)) return KTG_ERR_ARG;
        lap(ms[3]);
        parse_scl(pick(base, ".scl"), raw);
        lap(ms[4]);
        auto *b = new ktg_bookshelf();
        flatten(raw, *b);
        lap(ms[5]);
        std::copy(ms, ms + 6, b->ms);
        *out = b;
        return KTG_OK;
    } catch (const std::bad_alloc &) {
        g_error = "out of host memory";
        return KTG_ERR_NOMEM;
    } catch (const std::exception &e) {
        g_error = e.what();
        return KTG_ERR_ARG;
    }
}

void ktg_bookshelf_free(ktg_bookshelf *b) { delete b; }

int ktg_bookshelf_times(const ktg_bookshelf *b, double *ms) {
    if (!b || !ms) return KTG_ERR_ARG;
    std::copy(b->ms, b->ms + 6, ms);
    return KTG_OK;
}

int ktg_bookshelf_sizes(const ktg_bookshelf *b, int64_t *sizes) {
    if (!b || !sizes) return KTG_ERR_ARG;
    sizes[0] = b->V;
    sizes[1] = b->n;
    sizes[2] = b->N;
    sizes[3] = b->P;
    sizes[4] = b->Pm;
    sizes[5] = b->num_fixed;
    sizes[6] = static_cast<int64_t>(b->obstacles.size() / 4);
    sizes[7] = static_cast<int64_t>(b->rows.size() / 5);
    sizes[8] = static_cast<int64_t>(b->subrows.size() / 3);
    return KTG_OK;
}

int ktg_bookshelf_view(const ktg_bookshelf *b, ktg_netlist_view *v) {
    if (!b || !v) return KTG_ERR_ARG;
    v->num_vertices = b->V;
    v->num_movable = b->n;
    v->num_nets = b->N;
    v->mov_vertex = b->mov_vertex.data();
    v->var_of_vertex = b->var_of_vertex.data();
    v->fixed_x = b->fixed_x.data();
    v->fixed_y = b->fixed_y.data();
    v->net_start = b->net_start.data();
    v->pin_cell = b->pin_cell.data();
    v->off_x = b->off_x.data();
    v->off_y = b->off_y.data();
    v->net_weight = b->net_weight.data();
    v->pin_start = b->pin_start.data();
    v->pin_net = b->pin_net.data();
    v->pin_q = b->pin_q.data();
    v->width = b->width.data();
    v->height = b->height.data();
    return KTG_OK;
}

int ktg_bookshelf_geometry(const ktg_bookshelf *b, double *die4, double *obstacles, double *rows,
                           double *subrows) {
    if (!b) return KTG_ERR_ARG;
    if (die4) std::memcpy(die4, b->die, sizeof(b->die));
    if (obstacles) std::copy(b->obstacles.begin(), b->obstacles.end(), obstacles);
    if (rows) std::copy(b->rows.begin(), b->rows.end(), rows);
    if (subrows) std::copy(b->subrows.begin(), b->subrows.end(), subrows);
    return KTG_OK;
}

}  // extern "C"
