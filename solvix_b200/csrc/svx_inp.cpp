// Fast path of the Abaqus .inp reader for linear-static decks: the
// reference's parse_inp (crates/solvix-io/src/parser.rs:87-1370) restated in
// C++ for the keywords a linear-static deck uses, producing the model that
// svx_resolve consumes (the load state of Model::load_state, lib.rs:388-403)
// and the same warnings, errors and line numbers.
//
// Subset: *HEADING, *NODE, *ELEMENT, *NSET, *ELSET (GENERATE), *MATERIAL,
// *ELASTIC, *SOLID SECTION, *STEP (OP=, NAME=), *STATIC, *BOUNDARY (OP=),
// *CLOAD (OP=), *END STEP, and every keyword the reference does not know
// (warned and skipped, parser.rs:1303-1313).  The keywords the reference
// gives other meanings (density, plasticity, thermal, dynamics, beams,
// contact, distributed loads) and *STEP, NLGEOM=YES make svx_inp_parse
// return SVX_UNSUPPORTED, so that the host falls back to the reference's
// own parser for that deck.  Numbers follow Rust's FromStr: u32 / usize
// digits with an optional '+', f64 in Rust's decimal grammar (and inf /
// infinity / nan), read correctly rounded.
#include <algorithm>
#include <cctype>
#include <charconv>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <optional>
#include <string>
#include <string_view>
#include <unordered_map>
#include <utility>
#include <vector>

#include "solvix_gpu.h"
#include "svx_text.h"

namespace {

struct ParseFail {
    int64_t line;
    std::string message;
};

struct Unsupported {
    int64_t line;
    std::string keyword;
};

struct Item {
    bool kw = false;
    int64_t line = 0;
    std::string name;                                         // keyword, lower case
    std::vector<std::pair<std::string, std::string>> params;  // keys lower case
    std::string_view text;                                    // data line, trimmed
    const std::string* param(const char* key) const {
        const std::string* v = nullptr;  // a later duplicate wins, as in a HashMap
        for (const auto& p : params)
            if (p.first == key) v = &p.second;
        return v;
    }
};

bool is_ws(char c) {
    return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

std::string_view trim(std::string_view s) {
    size_t a = 0, b = s.size();
    while (a < b && is_ws(s[a])) ++a;
    while (b > a && is_ws(s[b - 1])) --b;
    return s.substr(a, b - a);
}

std::string lower(std::string_view s) {
    std::string o(s);
    for (auto& c : o) c = char(std::tolower(static_cast<unsigned char>(c)));
    return o;
}

std::string upper(std::string_view s) {
    std::string o(s);
    for (auto& c : o) c = char(std::toupper(static_cast<unsigned char>(c)));
    return o;
}

// parser.rs:1373-1411: `**` comments and blank lines dropped; `*NAME, K=V`
// keyword lines; everything else a data line.  Lines as str::lines() splits
// them ("\n", a trailing "\r" removed), numbered from 1.
std::vector<Item> tokenize(std::string_view text) {
    std::vector<Item> items;
    int64_t line = 0;
    size_t pos = 0;
    while (pos < text.size()) {
        size_t nl = text.find('\n', pos);
        std::string_view raw = text.substr(pos, nl == std::string_view::npos ? text.size() - pos
                                                                             : nl - pos);
        pos = (nl == std::string_view::npos) ? text.size() : nl + 1;
        ++line;
        if (!raw.empty() && raw.back() == '\r') raw.remove_suffix(1);
        const std::string_view t = trim(raw);
        if (t.empty() || (t.size() >= 2 && t[0] == '*' && t[1] == '*')) continue;
        Item it;
        it.line = line;
        if (t[0] == '*') {
            const std::string_view body = t.substr(1);
            const size_t comma = body.find(',');
            it.kw = true;
            it.name = lower(trim(body.substr(0, comma)));
            if (comma != std::string_view::npos) {
                std::string_view rest = body.substr(comma + 1);
                size_t p0 = 0;
                while (p0 <= rest.size()) {
                    size_t c = rest.find(',', p0);
                    std::string_view p = trim(rest.substr(p0, c == std::string_view::npos
                                                                  ? rest.size() - p0
                                                                  : c - p0));
                    if (!p.empty()) {
                        const size_t eq = p.find('=');
                        if (eq == std::string_view::npos)
                            it.params.emplace_back(lower(p), std::string());
                        else
                            it.params.emplace_back(lower(trim(p.substr(0, eq))),
                                                   std::string(trim(p.substr(eq + 1))));
                    }
                    if (c == std::string_view::npos) break;
                    p0 = c + 1;
                }
            }
        } else {
            it.text = t;  // a view into the deck, which outlives the parse
        }
        items.push_back(std::move(it));
    }
    return items;
}

// parser.rs:1413-1419: comma-split, trimmed, trailing empty fields dropped.
std::vector<std::string_view> fields(std::string_view line) {
    std::vector<std::string_view> f;
    size_t p0 = 0;
    for (;;) {
        const size_t c = line.find(',', p0);
        f.push_back(trim(line.substr(p0, c == std::string_view::npos ? line.size() - p0
                                                                     : c - p0)));
        if (c == std::string_view::npos) break;
        p0 = c + 1;
    }
    while (!f.empty() && f.back().empty()) f.pop_back();
    return f;
}

// Rust's FromStr for unsigned integers: an optional '+', then digits only.
template <class T>
std::optional<T> parse_unsigned(std::string_view s) {
    if (!s.empty() && s[0] == '+') s.remove_prefix(1);
    if (s.empty()) return std::nullopt;
    unsigned long long v = 0;
    for (char c : s) {
        if (c < '0' || c > '9') return std::nullopt;
        const unsigned long long d = (unsigned long long)(c - '0');
        if (v > (~0ULL - d) / 10) return std::nullopt;
        v = v * 10 + d;
    }
    if (v > (unsigned long long)(T)(~T(0))) return std::nullopt;
    return T(v);
}

// Rust's FromStr for f64 (core::num::dec2flt): [+-] then inf / infinity /
// nan (any case) or digits[.digits] / .digits with an optional exponent
// e[+-]digits.  Once the grammar is checked, from_chars reads the value
// correctly rounded (it takes no '+', so the sign is applied here; strtod
// covers what it reports out of range, rounding to inf or 0 as Rust does).
std::optional<double> parse_f64(std::string_view s) {
    std::string_view b = s;
    bool neg = false;
    if (!b.empty() && (b[0] == '+' || b[0] == '-')) {
        neg = b[0] == '-';
        b.remove_prefix(1);
    }
    if (b.empty()) return std::nullopt;
    bool ok = false;
    if (std::isalpha(static_cast<unsigned char>(b[0]))) {
        const std::string lb = lower(b);
        ok = (lb == "inf" || lb == "infinity" || lb == "nan");
    } else {
        size_t i = 0, int_d = 0, frac_d = 0;
        auto digit = [&](size_t k) {
            return k < b.size() && std::isdigit(static_cast<unsigned char>(b[k]));
        };
        while (digit(i)) ++i, ++int_d;
        if (i < b.size() && b[i] == '.') {
            ++i;
            while (digit(i)) ++i, ++frac_d;
        }
        ok = (int_d + frac_d) > 0;
        if (ok && i < b.size() && (b[i] == 'e' || b[i] == 'E')) {
            ++i;
            if (i < b.size() && (b[i] == '+' || b[i] == '-')) ++i;
            size_t exp_d = 0;
            while (digit(i)) ++i, ++exp_d;
            ok = exp_d > 0;
        }
        ok = ok && i == b.size();
    }
    if (!ok) return std::nullopt;
    double v = 0.0;
    const auto r = std::from_chars(b.data(), b.data() + b.size(), v);
    if (r.ec != std::errc() || r.ptr != b.data() + b.size()) {
        const std::string z(b);
        v = std::strtod(z.c_str(), nullptr);
    }
    return neg ? -v : v;
}

template <class T>
T num_u(std::string_view s, int64_t line, const char* what) {
    const auto v = parse_unsigned<T>(s);
    if (!v) throw ParseFail{line, std::string("malformed ") + what + " '" + std::string(s) + "'"};
    return *v;
}

double num_f(std::string_view s, int64_t line, const char* what) {
    const auto v = parse_f64(s);
    if (!v) throw ParseFail{line, std::string("malformed ") + what + " '" + std::string(s) + "'"};
    return *v;
}

struct Bc {
    std::vector<uint32_t> nodes;
    std::vector<int64_t> dofs;
};
struct Cload {
    uint32_t node;
    int64_t dof;
    double value;
};
struct Dload {
    uint32_t elem;
    int64_t face;
    double magnitude;
};

struct Gravity {
    double g;
    double dir[3];
};

struct StepAcc {
    std::vector<Bc> bcs;
    std::vector<Cload> cloads;
    std::vector<Dload> dloads;
    std::optional<Gravity> gravity;
};

// parser.rs:176-185: the element types it knows, with their node counts
// (ElemKind::node_count) and the Debug names of its error texts.
struct KindInfo {
    const char* type;
    int kind;
    int nodes;
    const char* debug;
};
const KindInfo KINDS[] = {{"CPS4", SVX_CPS4, 4, "Cps4"}, {"CPS3", SVX_CPS3, 3, "Cps3"},
                          {"CPS8", SVX_CPS8, 8, "Cps8"}, {"CPE4", SVX_CPE4, 4, "Cpe4"},
                          {"CPE8", SVX_CPE8, 8, "Cpe8"}, {"C3D8", SVX_C3D8, 8, "C3d8"},
                          {"C3D4", SVX_C3D4, 4, "C3d4"}, {"B31", SVX_B31, 2, "B31"}};

// Keywords the reference gives a meaning outside the linear-static path.
bool outside_subset(const std::string& k) {
    static const char* names[] = {"plastic",      "conductivity", "expansion",
                                  "beam section", "surface",      "surface interaction",
                                  "friction",     "contact pair", "temperature",
                                  "dflux",        "cflux",        "heat transfer",
                                  "dynamic",      "damping"};
    for (const char* n : names)
        if (k == n) return true;
    return false;
}

}  // namespace

struct svx_inp {
    std::vector<uint32_t> node_ids;
    std::vector<double> coords;
    std::vector<uint32_t> elem_ids;
    std::vector<uint8_t> kinds;
    std::vector<int64_t> conn_ptr{0};
    std::vector<uint32_t> conn;
    std::vector<std::string> mat_names;
    std::vector<double> youngs, poisson;
    std::vector<std::string> elset_names;
    std::vector<std::vector<uint32_t>> elset_ids;
    std::vector<std::pair<std::string, std::string>> assign;
    double thickness = 1.0;
    double density = 7850.0;  // Model::default (lib.rs:310-317)
    StepAcc state;  // Model::load_state
    int32_t n_steps = 0;
    std::vector<std::string> warnings;
    // flattened views behind desc
    std::vector<const char*> p_mat, p_elset, p_assign_e, p_assign_m;
    std::vector<int64_t> elset_ptr;
    std::vector<uint32_t> elset_flat;
    std::vector<int64_t> bc_node_ptr, bc_dof_ptr, bc_dofs, cl_dofs;
    std::vector<uint32_t> bc_nodes, cl_nodes, dl_elems;
    std::vector<double> cl_values, dl_values;
    std::vector<int64_t> dl_faces;
    svx_model_desc_t desc{};

    void parse(std::string_view text);
    void finish();
};

void svx_inp::parse(std::string_view text) {
    const std::vector<Item> items = tokenize(text);
    std::unordered_map<std::string, std::vector<uint32_t>> nsets;
    std::unordered_map<std::string, size_t> elset_index;
    std::unordered_map<uint32_t, char> node_seen;
    std::unordered_map<uint32_t, int> elem_kind;  // element id -> kind
    std::optional<std::string> pending_material, cur_material;
    bool density_seen = false;
    StepAcc model_data;
    std::vector<StepAcc> steps_done;
    std::optional<StepAcc> cur;
    int64_t step_no = 0;
    auto warn = [&](std::string w) { warnings.push_back(std::move(w)); };
    auto L = [](int64_t l) { return "line " + std::to_string(l) + ": "; };
    auto upsert_elset = [&](const std::string& name, const uint32_t* ids, size_t n) {
        const std::string key = upper(name);  // parser.rs:1495-1506
        auto it = elset_index.find(key);
        if (it == elset_index.end()) {
            elset_index.emplace(key, elset_names.size());
            elset_names.push_back(key);
            elset_ids.emplace_back(ids, ids + n);
        } else {
            auto& v = elset_ids[it->second];
            v.insert(v.end(), ids, ids + n);
        }
    };
    // parser.rs:1433-1449: node set first, then a bare node id
    auto resolve_nodes = [&](std::string_view target, int64_t line) {
        auto it = nsets.find(upper(target));
        if (it != nsets.end()) return it->second;
        const auto id = parse_unsigned<uint32_t>(target);
        if (!id) throw ParseFail{line, "unknown node set '" + std::string(target) + "'"};
        return std::vector<uint32_t>{*id};
    };
    // parser.rs:71-85
    auto op_is_new = [&](const Item& kw) {
        const std::string* v = kw.param("op");
        if (!v) return false;
        const std::string lv = lower(*v);
        if (lv == "new") return true;
        if (lv == "mod") return false;
        warn(L(kw.line) + "unsupported OP='" + lv + "' on *" + upper(kw.name) +
             " — treated as MOD");
        return false;
    };
    size_t j = 0;
    auto skip_data = [&] {
        while (j < items.size() && !items[j].kw) ++j;
    };
    while (j < items.size()) {
        const Item& kw = items[j];
        if (!kw.kw) {
            warn(L(kw.line) + "data line outside any keyword block ignored");
            ++j;
            continue;
        }
        if (pending_material) {
            static const char* mat_kws[] = {"elastic",   "density", "conductivity",
                                            "expansion", "damping", "plastic"};
            bool ok = false;
            for (const char* m : mat_kws) ok |= (kw.name == m);
            if (!ok) {
                warn(L(kw.line) + "material '" + *pending_material + "' has no *ELASTIC block");
                pending_material.reset();
            }
        }
        const std::string& name = kw.name;
        if (outside_subset(name)) throw Unsupported{kw.line, upper(name)};
        if (name == "heading") {
            ++j;
            skip_data();
        } else if (name == "node") {  // parser.rs:146-173
            ++j;
            for (; j < items.size() && !items[j].kw; ++j) {
                const Item& d = items[j];
                const auto f = fields(d.text);
                if (f.size() != 3 && f.size() != 4)
                    throw ParseFail{d.line, "*NODE expects id, x, y[, z]; got " +
                                                std::to_string(f.size()) + " field(s)"};
                const uint32_t id = num_u<uint32_t>(f[0], d.line, "node id");
                const double x = num_f(f[1], d.line, "coordinate");
                const double y = num_f(f[2], d.line, "coordinate");
                const double z = f.size() == 4 ? num_f(f[3], d.line, "coordinate") : 0.0;
                if (!node_seen.emplace(id, 1).second)
                    throw ParseFail{d.line, "duplicate node id " + std::to_string(id)};
                node_ids.push_back(id);
                coords.insert(coords.end(), {x, y, z});
            }
        } else if (name == "element") {  // parser.rs:175-256
            const std::string* ty = kw.param("type");
            const KindInfo* k = nullptr;
            if (ty) {
                const std::string t = upper(*ty);
                for (const auto& ki : KINDS)
                    if (t == ki.type) k = &ki;
            }
            if (!k) {
                const std::string what =
                    ty ? "element TYPE=" + upper(*ty) : std::string("TYPE-less *ELEMENT");
                warn(L(kw.line) + "unsupported " + what +
                     " — block skipped (supported: CPS3/CPS4/CPS8/CPE4/CPE8/C3D8/C3D4/B31)");
                ++j;
                skip_data();
                continue;
            }
            const size_t want = 1 + size_t(k->nodes);
            const std::string* setname = kw.param("elset");
            ++j;
            while (j < items.size() && !items[j].kw) {
                // one element per record; a trailing comma continues it
                std::vector<std::string> f;
                int64_t first = 0;
                while (j < items.size() && !items[j].kw) {
                    const Item& d = items[j];
                    if (f.empty()) first = d.line;
                    const bool ends_comma = !d.text.empty() && d.text.back() == ',';
                    std::string_view t = d.text;
                    size_t p0 = 0;
                    for (;;) {
                        const size_t c = t.find(',', p0);
                        f.emplace_back(trim(t.substr(p0, c == std::string_view::npos
                                                             ? t.size() - p0
                                                             : c - p0)));
                        if (c == std::string_view::npos) break;
                        p0 = c + 1;
                    }
                    ++j;
                    size_t have = 0;
                    for (const auto& x : f) have += !x.empty();
                    if (!ends_comma || have >= want) break;
                }
                std::vector<std::string> g;
                for (auto& x : f)
                    if (!x.empty()) g.push_back(std::move(x));
                if (g.size() != want)
                    throw ParseFail{first, std::string("*ELEMENT ") + k->debug + " expects " +
                                               std::to_string(want) + " field(s) (id + " +
                                               std::to_string(want - 1) + " nodes); got " +
                                               std::to_string(g.size())};
                const uint32_t id = num_u<uint32_t>(g[0], first, "element id");
                std::vector<uint32_t> c;
                for (size_t q = 1; q < g.size(); ++q)
                    c.push_back(num_u<uint32_t>(g[q], first, "node id"));
                if (!elem_kind.emplace(id, k->kind).second)
                    throw ParseFail{first, "duplicate element id " + std::to_string(id)};
                if (setname) upsert_elset(*setname, &id, 1);
                elem_ids.push_back(id);
                kinds.push_back(uint8_t(k->kind));
                conn.insert(conn.end(), c.begin(), c.end());
                conn_ptr.push_back(int64_t(conn.size()));
            }
        } else if (name == "elset" || name == "nset") {  // parser.rs:258-312
            const std::string* nm = kw.param("elset");
            if (!nm) nm = kw.param("nset");
            const bool generate = kw.param("generate") != nullptr;
            if (!nm) {
                warn(L(kw.line) + "set keyword without ELSET=/NSET= name — block skipped");
                ++j;
                skip_data();
                continue;
            }
            const std::string set = upper(*nm);
            ++j;
            for (; j < items.size() && !items[j].kw; ++j) {
                const Item& d = items[j];
                const auto f = fields(d.text);
                std::vector<uint32_t> ids;
                if (generate) {
                    if (f.size() < 2 || f.size() > 3)
                        throw ParseFail{d.line, "GENERATE expects start, end[, step]; got " +
                                                    std::to_string(f.size()) + " field(s)"};
                    const uint32_t a = num_u<uint32_t>(f[0], d.line, "set id");
                    const uint32_t b = num_u<uint32_t>(f[1], d.line, "set id");
                    const uint32_t st = f.size() == 3 ? num_u<uint32_t>(f[2], d.line, "set step")
                                                      : 1u;
                    if (st == 0) throw ParseFail{d.line, "GENERATE step must be >= 1"};
                    for (uint64_t v = a; v <= b; v += st) ids.push_back(uint32_t(v));
                } else {
                    for (const auto& x : f) ids.push_back(num_u<uint32_t>(x, d.line,
                                                                          "set member id"));
                }
                if (name == "elset") {
                    upsert_elset(set, ids.data(), ids.size());
                } else {
                    auto& v = nsets[set];
                    v.insert(v.end(), ids.begin(), ids.end());
                }
            }
        } else if (name == "material") {  // parser.rs:314-330
            const std::string* nm = kw.param("name");
            if (nm) {
                pending_material = upper(*nm);
                cur_material = upper(*nm);
            } else {
                warn(L(kw.line) + "*MATERIAL without NAME — block ignored");
            }
            ++j;
            skip_data();
        } else if (name == "elastic") {  // parser.rs:496-535
            ++j;
            bool got_row = false;
            for (; j < items.size() && !items[j].kw; ++j) {
                const Item& d = items[j];
                const auto f = fields(d.text);
                if (!got_row) {
                    if (f.size() != 2)
                        throw ParseFail{d.line,
                                        "*ELASTIC expects youngs_modulus, poisson_ratio; got " +
                                            std::to_string(f.size()) + " field(s)"};
                    if (pending_material) {
                        const std::string nm = *pending_material;
                        pending_material.reset();
                        const double e = num_f(f[0], d.line, "youngs modulus");
                        const double nu = num_f(f[1], d.line, "poisson ratio");
                        mat_names.push_back(nm);
                        youngs.push_back(e);
                        poisson.push_back(nu);
                    } else {
                        warn(L(d.line) + "*ELASTIC outside *MATERIAL — block ignored");
                    }
                    got_row = true;
                } else {
                    warn(L(d.line) +
                         "extra *ELASTIC row ignored (temperature dependence is v0.2)");
                }
            }
        } else if (name == "density") {  // parser.rs:332-365
            ++j;
            bool first_row = true;
            for (; j < items.size() && !items[j].kw; ++j) {
                const Item& d = items[j];
                const auto f = fields(d.text);
                if (first_row) {
                    if (!cur_material) {
                        warn(L(d.line) + "*DENSITY outside *MATERIAL — ignored");
                    } else if (f.empty()) {
                        throw ParseFail{d.line, "*DENSITY expects a density value"};
                    } else {
                        const double v = num_f(f[0], d.line, "density");
                        if (density_seen && density != v)
                            warn(L(d.line) + "*DENSITY overwrites an earlier value "
                                             "(per-material density is v0.4)");
                        density = v;
                        density_seen = true;
                        if (f.size() > 1)
                            warn(L(d.line) + "extra *DENSITY fields ignored (temperature "
                                             "dependence is v0.2)");
                    }
                    first_row = false;
                } else {
                    warn(L(d.line) +
                         "extra *DENSITY row ignored (temperature dependence is v0.2)");
                }
            }
        } else if (name == "dload") {  // parser.rs:846-950
            const bool op_new = op_is_new(kw);
            if (!cur) {
                warn(L(kw.line) +
                     "*DLOAD outside *STEP — ignored (distributed loads live in steps)");
                ++j;
                skip_data();
                continue;
            }
            if (op_new) {
                cur->dloads.clear();
                cur->gravity.reset();
            }
            ++j;
            for (; j < items.size() && !items[j].kw; ++j) {
                const Item& d = items[j];
                const auto f = fields(d.text);
                if (!f.empty() && lower(f[0]) == "grav") {
                    if (f.size() < 3 || f.size() > 5)
                        throw ParseFail{d.line, "*DLOAD GRAV expects GRAV, magnitude, dir1[, "
                                                "dir2][, dir3]; got " +
                                                    std::to_string(f.size()) + " field(s)"};
                    Gravity gr{};
                    gr.g = num_f(f[1], d.line, "gravity magnitude");
                    gr.dir[0] = num_f(f[2], d.line, "gravity direction");
                    gr.dir[1] = f.size() > 3 ? num_f(f[3], d.line, "gravity direction") : 0.0;
                    gr.dir[2] = f.size() > 4 ? num_f(f[4], d.line, "gravity direction") : 0.0;
                    cur->gravity = gr;
                    continue;
                }
                if (f.size() != 3)
                    throw ParseFail{d.line,
                                    "*DLOAD expects element/elset, P1..P4, magnitude; got " +
                                        std::to_string(f.size()) + " field(s)"};
                const std::string ltype = upper(f[1]);
                std::optional<uint64_t> face;
                if (!ltype.empty() && ltype[0] == 'P')
                    face = parse_unsigned<uint64_t>(std::string_view(ltype).substr(1));
                if (!face || *face < 1 || *face > 4) {
                    warn(L(d.line) + "*DLOAD type '" + ltype +
                         "' unsupported (v0.3: P1|P2|P3|P4, GRAV) — line ignored");
                    continue;
                }
                const double magnitude = num_f(f[2], d.line, "pressure magnitude");
                // parser.rs:1450-1457: an element set first, then a bare id
                std::vector<uint32_t> ids;
                const auto es = elset_index.find(upper(f[0]));
                if (es != elset_index.end()) {
                    ids = elset_ids[es->second];
                } else if (const auto id = parse_unsigned<uint32_t>(f[0])) {
                    ids.push_back(*id);
                } else {
                    warn(L(d.line) + "*DLOAD target '" + std::string(f[0]) +
                         "' is not a known element or ELSET — line ignored");
                    continue;
                }
                for (const uint32_t id : ids) {
                    const auto ek = elem_kind.find(id);
                    if (ek == elem_kind.end()) {
                        warn(L(d.line) + "*DLOAD on unknown element " + std::to_string(id) +
                             " — ignored");
                        continue;
                    }
                    const int kind = ek->second;
                    const uint64_t faces =
                        kind == SVX_CPS3 ? 3 : ((kind == SVX_CPS4 || kind == SVX_CPE4) ? 4 : 0);
                    if (*face > faces) {
                        std::string kn;
                        for (const auto& ki : KINDS)
                            if (ki.kind == kind) kn = lower(ki.type);
                        warn(L(d.line) + "element " + std::to_string(id) + " (" + kn +
                             ") has no face " + std::to_string(*face) + " — ignored");
                        continue;
                    }
                    cur->dloads.push_back(Dload{id, int64_t(*face), magnitude});
                }
            }
        } else if (name == "solid section") {  // parser.rs:537-584
            const std::string* es = kw.param("elset");
            const std::string* ms = kw.param("material");
            ++j;
            if (es && ms) {
                const std::string e = upper(*es), m = upper(*ms);
                if (!elset_index.count(e))
                    throw ParseFail{kw.line, "*SOLID SECTION references unknown ELSET '" + e + "'"};
                if (std::find(mat_names.begin(), mat_names.end(), m) == mat_names.end())
                    throw ParseFail{kw.line,
                                    "*SOLID SECTION references unknown MATERIAL '" + m + "'"};
                assign.emplace_back(e, m);
                if (j < items.size() && !items[j].kw) {
                    const Item& d = items[j];
                    const auto f = fields(d.text);
                    if (f.size() != 1)
                        throw ParseFail{d.line,
                                        "*SOLID SECTION data expects one thickness; got " +
                                            std::to_string(f.size()) + " field(s)"};
                    thickness = num_f(f[0], d.line, "thickness");
                    ++j;
                }
                skip_data();
            } else {
                warn(L(kw.line) + "*SOLID SECTION needs ELSET and MATERIAL — block skipped");
                skip_data();
            }
        } else if (name == "boundary" || name == "cload") {  // parser.rs:742-844
            const bool is_bc = name == "boundary";
            bool op_new = op_is_new(kw);
            if (!cur) {
                if (op_new) {
                    warn(L(kw.line) + "OP=NEW outside *STEP ignored");
                    op_new = false;
                }
                if (!steps_done.empty())
                    warn(L(kw.line) + (is_bc ? "*BOUNDARY" : "*CLOAD") +
                         " between steps — ignored");
            } else if (op_new) {
                if (is_bc)
                    cur->bcs.clear();
                else
                    cur->cloads.clear();
            }
            StepAcc& acc = cur ? *cur : model_data;
            ++j;
            for (; j < items.size() && !items[j].kw; ++j) {
                const Item& d = items[j];
                const auto f = fields(d.text);
                if (is_bc) {
                    if (f.size() < 2 || f.size() > 4)
                        throw ParseFail{d.line,
                                        "*BOUNDARY expects node/set, dof[, dof][, value]; got " +
                                            std::to_string(f.size()) + " field(s)"};
                    Bc bc;
                    bc.nodes = resolve_nodes(f[0], d.line);
                    const uint64_t d1 = num_u<uint64_t>(f[1], d.line, "dof");
                    if (f.size() >= 3) {
                        const uint64_t d2 = num_u<uint64_t>(f[2], d.line, "dof");
                        for (uint64_t v = d1; v <= d2 && v >= d1; ++v) {
                            bc.dofs.push_back(int64_t(v));
                            if (v == ~0ULL) break;
                        }
                    } else {
                        bc.dofs.push_back(int64_t(d1));
                    }
                    if (f.size() == 4) {
                        const double value = num_f(f[3], d.line, "prescribed value");
                        if (value != 0.0) {
                            std::string w = L(d.line) + "nonzero prescribed displacement ";
                            svx::rust_display_f64(w, value);
                            w += " ignored (v0.1: homogeneous BCs only)";
                            warn(std::move(w));
                        }
                    }
                    acc.bcs.push_back(std::move(bc));
                } else {
                    if (f.size() != 3)
                        throw ParseFail{d.line, "*CLOAD expects node/set, dof, value; got " +
                                                    std::to_string(f.size()) + " field(s)"};
                    const auto nodes = resolve_nodes(f[0], d.line);
                    const uint64_t dof = num_u<uint64_t>(f[1], d.line, "dof");
                    const double value = num_f(f[2], d.line, "load value");
                    for (uint32_t nid : nodes)
                        acc.cloads.push_back(Cload{nid, int64_t(dof), value});
                }
            }
        } else if (name == "step") {  // parser.rs:1114-1160
            if (cur) {
                steps_done.push_back(std::move(*cur));
                cur.reset();
            }
            ++step_no;
            bool op_new = false;
            if (const std::string* v = kw.param("op")) {
                const std::string lv = lower(*v);
                if (lv == "new")
                    op_new = true;
                else if (lv != "mod")
                    warn(L(kw.line) + "unsupported OP='" + lv + "' on *STEP — treated as MOD");
            }
            if (const std::string* v = kw.param("nlgeom")) {
                const std::string lv = lower(*v);
                if (lv == "yes" || lv.empty()) throw Unsupported{kw.line, "STEP, NLGEOM=YES"};
                if (lv != "no")
                    warn(L(kw.line) + "unsupported NLGEOM='" + lv + "' on *STEP — treated as NO");
            }
            cur = op_new ? StepAcc{} : (steps_done.empty() ? model_data : steps_done.back());
            ++j;
            skip_data();
        } else if (name == "static") {  // parser.rs:1279-1290
            if (!kw.params.empty())
                warn(L(kw.line) + "*STATIC parameters ignored (v0.1: linear static only)");
            ++j;
            skip_data();
        } else if (name == "end step") {  // parser.rs:1292-1300
            if (cur) {
                steps_done.push_back(std::move(*cur));
                cur.reset();
            }
            ++j;
            skip_data();
        } else {  // parser.rs:1303-1313
            warn(L(kw.line) + "unsupported keyword '*" + upper(name) + "' — block skipped");
            ++j;
            skip_data();
        }
    }
    if (pending_material) warn("material '" + *pending_material + "' has no *ELASTIC block");
    if (cur) {
        steps_done.push_back(std::move(*cur));
        cur.reset();
    }
    n_steps = int32_t(steps_done.size());
    // Model::load_state: the last step's accumulated state, else the
    // step-less deck's own BCs and loads
    state = steps_done.empty() ? std::move(model_data) : std::move(steps_done.back());
}

void svx_inp::finish() {
    for (const auto& s : mat_names) p_mat.push_back(s.c_str());
    for (const auto& s : elset_names) p_elset.push_back(s.c_str());
    elset_ptr.assign(1, 0);
    for (const auto& v : elset_ids) {
        elset_flat.insert(elset_flat.end(), v.begin(), v.end());
        elset_ptr.push_back(int64_t(elset_flat.size()));
    }
    for (const auto& a : assign) {
        p_assign_e.push_back(a.first.c_str());
        p_assign_m.push_back(a.second.c_str());
    }
    bc_node_ptr.assign(1, 0);
    bc_dof_ptr.assign(1, 0);
    for (const auto& b : state.bcs) {
        bc_nodes.insert(bc_nodes.end(), b.nodes.begin(), b.nodes.end());
        bc_dofs.insert(bc_dofs.end(), b.dofs.begin(), b.dofs.end());
        bc_node_ptr.push_back(int64_t(bc_nodes.size()));
        bc_dof_ptr.push_back(int64_t(bc_dofs.size()));
    }
    for (const auto& c : state.cloads) {
        cl_nodes.push_back(c.node);
        cl_dofs.push_back(c.dof);
        cl_values.push_back(c.value);
    }
    for (const auto& dl : state.dloads) {
        dl_elems.push_back(dl.elem);
        dl_faces.push_back(dl.face);
        dl_values.push_back(dl.magnitude);
    }
    svx_model_desc_t& d = desc;
    d.n_nodes = int64_t(node_ids.size());
    d.node_ids = node_ids.data();
    d.node_coords = coords.data();
    d.n_elems = int64_t(elem_ids.size());
    d.elem_ids = elem_ids.data();
    d.elem_kinds = kinds.data();
    d.elem_conn_ptr = conn_ptr.data();
    d.elem_conn = conn.data();
    d.n_materials = int32_t(mat_names.size());
    d.material_names = p_mat.data();
    d.youngs_modulus = youngs.data();
    d.poisson_ratio = poisson.data();
    d.n_elsets = int32_t(elset_names.size());
    d.elset_names = p_elset.data();
    d.elset_ptr = elset_ptr.data();
    d.elset_elem_ids = elset_flat.data();
    d.n_assignments = int32_t(assign.size());
    d.assign_elset = p_assign_e.data();
    d.assign_material = p_assign_m.data();
    d.thickness = thickness;
    d.n_bcs = int32_t(state.bcs.size());
    d.bc_node_ptr = bc_node_ptr.data();
    d.bc_node_ids = bc_nodes.data();
    d.bc_dof_ptr = bc_dof_ptr.data();
    d.bc_dofs = bc_dofs.data();
    d.n_cloads = int64_t(cl_nodes.size());
    d.cload_node_ids = cl_nodes.data();
    d.cload_dofs = cl_dofs.data();
    d.cload_values = cl_values.data();
    d.density = density;
    d.n_dloads = int64_t(dl_elems.size());
    d.dload_elem_ids = dl_elems.data();
    d.dload_faces = dl_faces.data();
    d.dload_values = dl_values.data();
    d.has_gravity = state.gravity ? 1 : 0;
    if (state.gravity) {
        d.gravity_magnitude = state.gravity->g;
        for (int k = 0; k < 3; ++k) d.gravity_dir[k] = state.gravity->dir[k];
    }
}

namespace {

void put_error(svx_error_t* err, int code, int64_t line, const std::string& msg) {
    if (!err) return;
    std::memset(err, 0, sizeof(*err));
    err->code = code;
    err->elem_index = line;
    std::snprintf(err->message, sizeof(err->message), "%s", msg.c_str());
}

}  // namespace

extern "C" {

int svx_inp_parse(const char* text, int64_t len, svx_inp_t** out, svx_error_t* err) {
    if (!out || (!text && len > 0) || len < 0) {
        put_error(err, SVX_BAD_ARGUMENT, -1, "bad argument");
        return SVX_BAD_ARGUMENT;
    }
    *out = nullptr;
    try {
        std::unique_ptr<svx_inp> p(new svx_inp());
        p->parse(std::string_view(text ? text : "", size_t(len)));
        p->finish();
        put_error(err, SVX_OK, -1, "");
        *out = p.release();
        return SVX_OK;
    } catch (const ParseFail& f) {
        put_error(err, SVX_PARSE_ERROR, f.line, f.message);
        return SVX_PARSE_ERROR;
    } catch (const Unsupported& u) {
        put_error(err, SVX_UNSUPPORTED, u.line,
                  "line " + std::to_string(u.line) + ": *" + u.keyword +
                      " is outside the linear-static reader; parse this deck with the "
                      "reference parser");
        return SVX_UNSUPPORTED;
    } catch (const std::bad_alloc&) {
        put_error(err, SVX_OOM, -1, "host allocation failed");
        return SVX_OOM;
    }
}

const svx_model_desc_t* svx_inp_model(const svx_inp_t* inp) { return inp ? &inp->desc : nullptr; }

int32_t svx_inp_step_count(const svx_inp_t* inp) { return inp ? inp->n_steps : 0; }

int32_t svx_inp_warning_count(const svx_inp_t* inp) {
    return inp ? int32_t(inp->warnings.size()) : 0;
}

const char* svx_inp_warning(const svx_inp_t* inp, int32_t i) {
    if (!inp || i < 0 || i >= int32_t(inp->warnings.size())) return nullptr;
    return inp->warnings[size_t(i)].c_str();
}

void svx_inp_free(svx_inp_t* inp) { delete inp; }

}  // extern "C"
