// Structure input for compute_surface: PDB and mmCIF atom records, the
// default atom selection and element van der Waals radii, restating
// sesmesh's io/pdb.rs:139-300, io/cif/{lexer.rs,mod.rs} (the _atom_site
// loop), structure/select.rs:140-360 (model, alternate locations,
// hydrogens, waters, hetero atoms), structure/element.rs:86-168 (symbols and
// the atom-name rule) and radii/tables.rs:24-80 with radii/mod.rs:166-250
// (Bondi / Mantina radii, 1.80 A for elements without one).  Host code only:
// it turns file bytes into the (x, y, z, r) rows the mesh stage takes.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../../include/sesmesh_b200_surface.h"

namespace {

void set_err(char* err, size_t len, const char* fmt, ...) {
    if (!err || !len) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, len, fmt, ap);
    va_end(ap);
}

// Element symbols by atomic number (1..118).
const char* const SYMBOLS[119] = {
    "",   "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si", "P",  "S",
    "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As",
    "Se", "Br", "Kr", "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn",
    "Sb", "Te", "I",  "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho",
    "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W",  "Re", "Os", "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po",
    "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa", "U",  "Np", "Pu", "Am", "Cm", "Bk", "Cf", "Es", "Fm", "Md",
    "No", "Lr", "Rf", "Db", "Sg", "Bh", "Hs", "Mt", "Ds", "Rg", "Cn", "Nh", "Fl", "Mc", "Lv", "Ts", "Og"};

// The Bondi set (radii/tables.rs:24-80): Bondi 1964, completed with Mantina
// 2009 and the Bondi column of Alvarez 2013 (Z, radius in A).
const std::pair<int, double> BONDI[] = {
    {1, 1.20},  {2, 1.40},  {3, 1.81},  {4, 1.53},  {5, 1.92},  {6, 1.70},  {7, 1.55},  {8, 1.52},
    {9, 1.47},  {10, 1.54}, {11, 2.27}, {12, 1.73}, {13, 1.84}, {14, 2.10}, {15, 1.80}, {16, 1.80},
    {17, 1.75}, {18, 1.88}, {19, 2.75}, {20, 2.31}, {28, 1.63}, {29, 1.40}, {30, 1.39}, {31, 1.87},
    {32, 2.11}, {33, 1.85}, {34, 1.90}, {35, 1.83}, {36, 2.02}, {37, 3.03}, {38, 2.49}, {46, 1.63},
    {47, 1.72}, {48, 1.62}, {49, 1.93}, {50, 2.17}, {51, 2.06}, {52, 2.06}, {53, 1.98}, {54, 2.16},
    {55, 3.43}, {56, 2.68}, {78, 1.72}, {79, 1.66}, {80, 1.70}, {81, 1.96}, {82, 2.02}, {83, 2.07},
    {84, 1.97}, {85, 2.02}, {86, 2.20}, {87, 3.48}, {88, 2.83}, {92, 1.86}};
constexpr double UNKNOWN_RADIUS = 1.80;  // RadiusOptions::default (radii/mod.rs:155-163)

// Element::lookup (element.rs:106-121): case-insensitive symbol; one-letter
// D and T are hydrogen.  0: none.
int element_of(const char* s, size_t n) {
    while (n && std::isspace((unsigned char)*s)) s++, n--;
    while (n && std::isspace((unsigned char)s[n - 1])) n--;
    if (n < 1 || n > 2) return 0;
    const char a = char(std::toupper((unsigned char)s[0]));
    if (a < 'A' || a > 'Z') return 0;
    if (n == 1 && (a == 'D' || a == 'T')) return 1;
    char b = 0;
    if (n == 2) {
        if (!std::isalpha((unsigned char)s[1])) return 0;
        b = char(std::tolower((unsigned char)s[1]));
    }
    for (int z = 1; z <= 118; z++) {
        const char* sym = SYMBOLS[z];
        if (sym[0] == a && (n == 1 ? sym[1] == 0 : sym[1] == b)) return z;
    }
    return 0;
}

// Element::infer_from_name (element.rs:151-168): the letters of the atom name
// after leading non-letters; a two-letter element when the residue is named
// after it, the atom is a hetero heavy atom, or the first letter alone is no
// element; else the first letter.
int infer_element(const std::string& name, const std::string& res, bool het) {
    size_t i = 0;
    while (i < name.size() && !std::isalpha((unsigned char)name[i])) i++;
    std::string letters;
    while (i < name.size() && std::isalpha((unsigned char)name[i])) letters += name[i++];
    if (letters.empty()) return 0;
    if (letters.size() >= 2) {
        const int two = element_of(letters.data(), 2);
        if (two) {
            std::string r = res;
            while (!r.empty() && std::isspace((unsigned char)r.back())) r.pop_back();
            while (!r.empty() && std::isspace((unsigned char)r.front())) r.erase(r.begin());
            const char* sym = SYMBOLS[two];
            bool named_after = r.size() == std::strlen(sym);
            for (size_t k = 0; named_after && k < r.size(); k++)
                named_after = std::tolower((unsigned char)r[k]) == std::tolower((unsigned char)sym[k]);
            const bool hetero_heavy = het && std::toupper((unsigned char)letters[0]) != 'H';
            if (named_after || hetero_heavy || !element_of(letters.data(), 1)) return two;
        }
    }
    return element_of(letters.data(), 1);
}

struct Atom {
    double x, y, z;
    int element = 0;
    bool het = false;
    char alt = 0;  // 0: none
    float occupancy = 1.0f;
    std::string name, res, chain, label_chain;
    int seq = 0;
    char ins = 0;
};
struct Model {
    int number;
    std::vector<Atom> atoms;
};

std::string trim(const char* s, size_t n) {
    while (n && std::isspace((unsigned char)*s)) s++, n--;
    while (n && std::isspace((unsigned char)s[n - 1])) n--;
    return std::string(s, n);
}

bool parse_double(const std::string& t, double& v) {
    if (t.empty()) return false;
    // [+-]digits[.digits] with at most 15 digits (the fixed-point columns of
    // PDB and mmCIF coordinates): mantissa / 10^k, both exact in f64, so the
    // one division rounds the decimal value correctly, as strtod does.
    {
        size_t i = 0, nd = 0, frac = 0;
        bool neg = false, dot = false, ok = true;
        uint64_t mant = 0;
        if (t[0] == '+' || t[0] == '-') neg = t[0] == '-', i = 1;
        for (; i < t.size(); i++) {
            const char c = t[i];
            if (c >= '0' && c <= '9') {
                mant = mant * 10 + uint64_t(c - '0');
                nd++;
                if (dot) frac++;
            } else if (c == '.' && !dot) {
                dot = true;
            } else {
                ok = false;
                break;
            }
        }
        if (ok && nd > 0 && nd <= 15) {
            static const double P10[16] = {1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6, 1e7,
                                           1e8, 1e9, 1e10, 1e11, 1e12, 1e13, 1e14, 1e15};
            const double a = double(mant) / P10[frac];
            v = neg ? -a : a;
            return true;
        }
    }
    char* end = nullptr;
    v = std::strtod(t.c_str(), &end);
    return end == t.c_str() + t.size() && std::isfinite(v);
}

bool parse_int(const std::string& t, long long& v) {
    if (t.empty()) return false;
    char* end = nullptr;
    v = std::strtoll(t.c_str(), &end, 10);
    return end == t.c_str() + t.size();
}

// io/pdb.rs:139-300: ATOM / HETATM fixed columns, MODEL / ENDMDL / END.
std::string read_pdb(const char* data, size_t len, std::vector<Model>& models) {
    models.clear();
    int next_model = 1;
    bool in_model = false;
    size_t pos = 0, lineno = 0;
    auto model = [&]() -> Model& {
        if (!in_model) {
            models.push_back(Model{next_model++, {}});
            in_model = true;
        }
        return models.back();
    };
    while (pos < len) {
        lineno++;
        const char* nl = static_cast<const char*>(std::memchr(data + pos, '\n', len - pos));
        size_t end = nl ? size_t(nl - data) : len;
        std::string line(data + pos, end - pos);
        if (!line.empty() && line.back() == '\r') line.pop_back();
        pos = end + 1;
        const bool atom_rec = line.compare(0, 4, "ATOM") == 0 &&
                              (line.size() <= 4 || line[4] == ' ' || std::isdigit((unsigned char)line[4]));
        const bool het_rec = line.compare(0, 6, "HETATM") == 0;
        if (atom_rec || het_rec) {
            if (line.size() < 54) return "line " + std::to_string(lineno) + ": atom record too short for coordinates";
            Atom a;
            if (!parse_double(trim(line.data() + 30, 8), a.x) || !parse_double(trim(line.data() + 38, 8), a.y) ||
                !parse_double(trim(line.data() + 46, 8), a.z))
                return "line " + std::to_string(lineno) + ": invalid coordinates";
            auto col = [&](size_t s, size_t e) { return s >= line.size() ? std::string() : trim(line.data() + s, std::min(e, line.size()) - s); };
            auto ch = [&](size_t i) { return i < line.size() && line[i] != ' ' ? line[i] : char(0); };
            a.het = het_rec;
            a.name = col(12, 16);
            a.alt = ch(16);
            a.res = col(17, 21);
            a.chain = a.label_chain = col(21, 22);
            long long seq = 0;
            a.seq = parse_int(col(22, 26), seq) ? int(seq) : 0;
            a.ins = ch(26);
            const std::string occ = col(54, 60);
            double o;
            if (!occ.empty()) a.occupancy = parse_double(occ, o) ? float(o) : 1.0f;
            const std::string el = col(76, 78);
            a.element = el.empty() ? 0 : element_of(el.data(), el.size());
            if (!a.element) {
                const std::string raw = line.size() > 12 ? line.substr(12, std::min<size_t>(4, line.size() - 12)) : "";
                a.element = infer_element(raw, a.res, a.het);
            }
            model().atoms.push_back(std::move(a));
        } else if (line.compare(0, 6, "ENDMDL") == 0 || line.compare(0, 4, "END ") == 0 ||
                   (line.compare(0, 3, "END") == 0 && trim(line.data(), line.size()) == "END")) {
            in_model = false;
        } else if (line.compare(0, 5, "MODEL") == 0) {
            long long num = 0;
            const bool ok = parse_int(trim(line.data() + 5, line.size() - 5), num);
            models.push_back(Model{ok ? int(num) : next_model, {}});
            next_model = (ok ? int(num) : next_model) + 1;
            in_model = true;
        }
    }
    return "";
}

// io/cif/lexer.rs: whitespace-separated tokens, '...' / "..." quoted values
// (closed by the quote before whitespace), ;-delimited text fields, #
// comments.  Tokens keep a flag for values that are unquoted '.' or '?'.
struct Tok {
    std::string text;
    bool quoted = false;
};

void cif_tokens(const char* data, size_t len, std::vector<Tok>& out) {
    size_t i = 0;
    bool line_start = true;
    while (i < len) {
        const char c = data[i];
        if (c == '\n') {
            i++, line_start = true;
            continue;
        }
        if (std::isspace((unsigned char)c)) {
            i++;
            continue;
        }
        if (c == '#') {
            while (i < len && data[i] != '\n') i++;
            continue;
        }
        if (c == ';' && line_start) {
            size_t j = i + 1;
            std::string t;
            for (;;) {
                const char* nl = static_cast<const char*>(std::memchr(data + j, '\n', len - j));
                if (!nl) {
                    t.append(data + j, len - j), j = len;
                    break;
                }
                t.append(data + j, size_t(nl - data) - j + 1);
                j = size_t(nl - data) + 1;
                if (j < len && data[j] == ';') {
                    j++;
                    break;
                }
            }
            if (!t.empty() && t.back() == '\n') t.pop_back();
            out.push_back(Tok{t, true});
            i = j, line_start = false;
            continue;
        }
        line_start = false;
        if (c == '\'' || c == '"') {
            size_t j = i + 1;
            while (j < len && !(data[j] == c && (j + 1 >= len || std::isspace((unsigned char)data[j + 1])))) {
                if (data[j] == '\n') break;
                j++;
            }
            out.push_back(Tok{std::string(data + i + 1, j - i - 1), true});
            i = j < len && data[j] == c ? j + 1 : j;
            continue;
        }
        size_t j = i;
        while (j < len && !std::isspace((unsigned char)data[j])) j++;
        out.push_back(Tok{std::string(data + i, j - i), false});
        i = j;
    }
}

bool cif_is_null(const Tok& t) { return !t.quoted && (t.text == "." || t.text == "?"); }

std::string lower(std::string s) {
    for (char& c : s) c = char(std::tolower((unsigned char)c));
    return s;
}

// io/cif/mod.rs:20-420: the _atom_site loop of the first data block.
std::string read_cif(const char* data, size_t len, std::vector<Model>& models) {
    models.clear();
    std::vector<Tok> toks;
    cif_tokens(data, len, toks);
    size_t i = 0;
    for (; i < toks.size(); i++) {
        if (toks[i].quoted || lower(toks[i].text) != "loop_") continue;
        size_t j = i + 1;
        if (j < toks.size() && !toks[j].quoted && lower(toks[j].text).compare(0, 11, "_atom_site.") == 0) break;
    }
    if (i >= toks.size()) return "no _atom_site loop";
    std::map<std::string, size_t> col;
    size_t j = i + 1, ncol = 0;
    while (j < toks.size() && !toks[j].quoted && toks[j].text.size() > 11 &&
           lower(toks[j].text).compare(0, 11, "_atom_site.") == 0)
        col[lower(toks[j].text.substr(11))] = ncol++, j++;
    auto idx = [&](const char* name) -> long { auto it = col.find(name); return it == col.end() ? -1 : long(it->second); };
    const long cx = idx("cartn_x"), cy = idx("cartn_y"), cz = idx("cartn_z");
    if (cx < 0 || cy < 0 || cz < 0) return "_atom_site has no Cartn_x/y/z items";
    const long c_group = idx("group_pdb"), c_type = idx("type_symbol"), c_lname = idx("label_atom_id"),
               c_aname = idx("auth_atom_id"), c_alt = idx("label_alt_id"), c_lcomp = idx("label_comp_id"),
               c_acomp = idx("auth_comp_id"), c_lasym = idx("label_asym_id"), c_aasym = idx("auth_asym_id"),
               c_lseq = idx("label_seq_id"), c_aseq = idx("auth_seq_id"), c_ins = idx("pdbx_pdb_ins_code"),
               c_occ = idx("occupancy"), c_model = idx("pdbx_pdb_model_num");
    size_t last = 0;
    for (size_t row = j; row + ncol <= toks.size(); row += ncol) {
        // The loop ends at the next keyword or tag.
        const Tok& first = toks[row];
        if (!first.quoted && (first.text[0] == '_' || lower(first.text) == "loop_" ||
                              lower(first.text).compare(0, 5, "data_") == 0))
            break;
        auto get = [&](long c, std::string& out) -> bool {
            if (c < 0) return false;
            const Tok& t = toks[row + size_t(c)];
            if (cif_is_null(t)) return false;
            out = t.text;
            return true;
        };
        Atom a;
        std::string v;
        if (!get(cx, v) || !parse_double(v, a.x) || !get(cy, v) || !parse_double(v, a.y) || !get(cz, v) ||
            !parse_double(v, a.z))
            return "invalid _atom_site coordinates in row " + std::to_string((row - j) / ncol + 1);
        a.het = get(c_group, v) && lower(v) == "hetatm";
        if (!get(c_aname, a.name)) get(c_lname, a.name);
        if (get(c_alt, v) && !v.empty()) a.alt = v[0];
        if (!get(c_acomp, a.res)) get(c_lcomp, a.res);
        std::string lab;
        const bool has_lab = get(c_lasym, lab);
        if (!get(c_aasym, a.chain)) a.chain = has_lab ? lab : "";
        a.label_chain = has_lab ? lab : a.chain;
        long long seq = 0;
        if (get(c_aseq, v) || get(c_lseq, v)) a.seq = parse_int(v, seq) ? int(seq) : 0;
        if (get(c_ins, v) && !v.empty()) a.ins = v[0];
        double o;
        if (get(c_occ, v)) a.occupancy = parse_double(v, o) ? float(o) : 1.0f;
        if (get(c_type, v)) a.element = element_of(v.data(), v.size());
        if (!a.element) a.element = infer_element(a.name, a.res, a.het);
        long long mnum = 1;
        if (get(c_model, v) && !parse_int(v, mnum)) mnum = 1;
        if (models.empty() || models[last].number != int(mnum)) {
            last = models.size();
            for (size_t m = 0; m < models.size(); m++)
                if (models[m].number == int(mnum)) last = m;
            if (last == models.size()) models.push_back(Model{int(mnum), {}});
        }
        models[last].atoms.push_back(std::move(a));
    }
    return "";
}

bool is_water(const std::string& res) {
    static const char* const W[] = {"HOH", "DOD", "WAT", "H2O", "SOL", "TIP", "TIP3", "TIP4",
                                    "TIP5", "SPC", "T3P", "T4P", "T5P"};
    const std::string r = lower(res);
    for (const char* w : W)
        if (r == lower(w)) return true;
    return false;
}

double radius_of(int z) {
    for (const auto& p : BONDI)
        if (p.first == z) return p.second;
    return UNKNOWN_RADIUS;
}

}  // namespace

extern "C" int smb_read_structure(const char* data, size_t len, int format, const smb_selection* sel, double* xyzr,
                                  size_t cap, size_t* n, char* err, size_t errlen) {
    if (!data || !n) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    *n = 0;
    smb_selection S = sel ? *sel : smb_selection{0, 0, 0, 1};
    if (format == SMB_FORMAT_AUTO) {
        // mmCIF starts with a data_ block (after comments and blank lines).
        size_t i = 0;
        while (i < len) {
            while (i < len && std::isspace((unsigned char)data[i])) i++;
            if (i < len && data[i] == '#') {
                while (i < len && data[i] != '\n') i++;
                continue;
            }
            break;
        }
        format = (len - i >= 5 && std::strncmp(data + i, "data_", 5) == 0) ? SMB_FORMAT_MMCIF : SMB_FORMAT_PDB;
    }
    std::vector<Model> models;
    std::string m = format == SMB_FORMAT_MMCIF ? read_cif(data, len, models)
                    : format == SMB_FORMAT_PDB ? read_pdb(data, len, models)
                                               : std::string("unknown format");
    if (!m.empty()) return set_err(err, errlen, "%s", m.c_str()), SMB_ERR_ARG;
    // ModelChoice (select.rs:233-254): the first model, or by number.
    const Model* model = nullptr;
    for (const Model& md : models)
        if (S.model == 0 ? true : md.number == S.model) {
            model = &md;
            break;
        }
    if (!model) return set_err(err, errlen, "model %d not found", S.model), SMB_ERR_ARG;
    const std::vector<Atom>& atoms = model->atoms;
    // AltLocPolicy::HighestOccupancy (select.rs:298-370): per residue
    // (chain, number, insertion code, label chain), the letter of the highest
    // total occupancy, the first on ties.
    typedef std::tuple<std::string, int, char, std::string> Key;
    std::map<Key, std::vector<std::pair<char, double>>> letters;
    for (const Atom& a : atoms) {
        if (!a.alt) continue;
        auto& l = letters[Key(a.chain, a.seq, a.ins, a.label_chain)];
        auto it = std::find_if(l.begin(), l.end(), [&](const std::pair<char, double>& p) { return p.first == a.alt; });
        if (it == l.end()) l.push_back({a.alt, double(a.occupancy)});
        else it->second += double(a.occupancy);
    }
    std::map<Key, char> chosen;
    for (auto& kv : letters) {
        char best = kv.second[0].first;
        double occ = kv.second[0].second;
        for (size_t k = 1; k < kv.second.size(); k++)
            if (!(occ >= kv.second[k].second)) best = kv.second[k].first, occ = kv.second[k].second;
        chosen[kv.first] = best;
    }
    size_t count = 0;
    for (const Atom& a : atoms) {
        if (a.alt && chosen[Key(a.chain, a.seq, a.ins, a.label_chain)] != a.alt) continue;
        if (!S.hydrogens && a.element == 1) continue;
        if (!S.waters && is_water(a.res)) continue;
        if (!S.hetero && a.het) continue;
        if (xyzr && count < cap) {
            double* o = xyzr + 4 * count;
            o[0] = a.x, o[1] = a.y, o[2] = a.z, o[3] = radius_of(a.element);
        }
        count++;
    }
    *n = count;
    if (count == 0) return set_err(err, errlen, "no atom passed the selection"), SMB_ERR_ARG;
    if (xyzr && count > cap) return set_err(err, errlen, "%zu atoms do not fit in %zu", count, cap), SMB_ERR_MEMORY;
    return SMB_OK;
}
