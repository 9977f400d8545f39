/* dgsw_rkdg_problem.hpp - C++ host side of the drop-in, over the C ABI in dgsw_rkdg.h.
 *
 * Mirrors the reference's serial driver stack for the `rkdg_swe` problem:
 *   InputParameters        source/preprocessor/input_parameters.hpp:72-261 (the `.15` YAML file)
 *   SWE::Inputs            source/problem/SWE/problem_input/swe_inputs.{hpp:125-158, cpp:4-205}, read_bcis
 *                          (cpp:211-290), the Manning n file (swe_pre_init_data.hpp:165-182)
 *   AdcircFormat           source/preprocessor/ADCIRC_reader/adcirc_format.cpp:3-130, 214-254
 *   ESSPRKStepper queries  source/simulation/stepper/explicit_ssp_rk_stepper.hpp:36-65
 *   SWE::RKDG::Problem     source/problem/SWE/discretization_RKDG/rkdg_swe_problem.hpp:34-194
 *   Serial::Simulation     source/simulation/serial/simulation.hpp:14-93
 *   Writer                 source/simulation/writer.hpp:100-193 with the modal / VTK / VTU writers of
 *                          source/problem/SWE/problem_postprocessor/
 * so that a caller of SWE::RKDG::Problem / Serial::Simulation<SWE::RKDG::Problem> switches to
 * SWE::RKDG::GpuProblem / Serial::GpuSimulation<SWE::RKDG::GpuProblem>. All arithmetic of the step runs
 * in libdgsw_rkdg.so on the GPU; this header only parses input, owns the handle and forwards calls.
 *
 * Errors: input and mesh errors throw std::logic_error with the reference's messages where it has one;
 * library failures throw dgsw::Error carrying the dgsw_status and dgsw_last_error() text.
 *
 * Input extensions: the reference picks its analytic initial-condition / source / true-solution
 * functions at compile time (one example program per function set). Here a top-level `b200:` node of
 * the same `.15` file selects them at run time, together with the execution options; the reference's
 * parser ignores unknown top-level nodes, so one file serves both programs:
 *   b200:
 *     function_set: manufactured_sine   # none | reference_manufactured | manufactured_sine |
 *                                       # thacker_bowl | gaussian_humps
 *     function_parameters: [40000, 0.1, 2.0, 0.0, 9.81]
 *     precision: fp64                   # fp64 | fp32
 *     tile: 0                           # 0 = automatic, else 128 or 256
 *     device: 0
 */
#ifndef DGSW_RKDG_PROBLEM_HPP
#define DGSW_RKDG_PROBLEM_HPP

#include <time.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "dgsw_rkdg.h"

namespace dgsw {

/* ------------------------------------------------------------------------------------------------ */
/* errors                                                                                           */

class Error : public std::runtime_error {
  public:
    Error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
    int status() const { return status_; }

  private:
    int status_;
};

inline void check(int32_t status, const char* call) {
    if (status != DGSW_OK)
        throw Error(status, std::string(call) + ": " + dgsw_status_string(status) + ": " + dgsw_last_error());
}

/* ------------------------------------------------------------------------------------------------ */
/* YAML: the subset `.15` files use (block mappings by indentation, block and flow sequences of      */
/* scalars, comments, quoted scalars)                                                                */

class YamlNode {
  public:
    enum Kind { Null, Scalar, Map, Seq };

    Kind kind = Null;
    bool defined = false;  // present in the document, even with an empty value (yaml-cpp's IsDefined)
    std::string value;
    std::vector<std::pair<std::string, YamlNode>> map;
    std::vector<YamlNode> seq;

    explicit operator bool() const { return defined || kind != Null; }
    bool IsNull() const { return kind == Null || (kind == Scalar && (value.empty() || value == "~" || value == "null")); }

    const YamlNode& operator[](const std::string& key) const {
        static const YamlNode null_node;
        if (kind == Map)
            for (const auto& kv : map)
                if (kv.first == key) return kv.second;
        return null_node;
    }

    template <typename T>
    T as() const;

  private:
    [[noreturn]] void bad(const char* type) const {
        throw std::logic_error("Error: YAML value '" + value + "' is not a " + type + "\n");
    }
    friend YamlNode yaml_load(const std::string&);
};

template <>
inline std::string YamlNode::as<std::string>() const {
    if (kind != Scalar) bad("scalar");
    return value;
}
template <>
inline double YamlNode::as<double>() const {
    if (kind != Scalar) bad("number");
    char* end = nullptr;
    const double v = std::strtod(value.c_str(), &end);
    if (end == value.c_str() || *end != '\0') bad("number");
    return v;
}
template <>
inline long YamlNode::as<long>() const {
    if (kind != Scalar) bad("integer");
    char* end = nullptr;
    const long v = std::strtol(value.c_str(), &end, 10);
    if (end == value.c_str() || *end != '\0') bad("integer");
    return v;
}
template <>
inline int YamlNode::as<int>() const {
    return (int)as<long>();
}
template <>
inline unsigned YamlNode::as<unsigned>() const {
    const long v = as<long>();
    if (v < 0) bad("non-negative integer");
    return (unsigned)v;
}
template <>
inline bool YamlNode::as<bool>() const {
    if (kind != Scalar) bad("boolean");
    if (value == "true" || value == "True" || value == "TRUE" || value == "yes" || value == "on") return true;
    if (value == "false" || value == "False" || value == "FALSE" || value == "no" || value == "off") return false;
    bad("boolean");
}
template <>
inline std::vector<double> YamlNode::as<std::vector<double>>() const {
    std::vector<double> out;
    if (kind == Seq)
        for (const auto& n : seq) out.push_back(n.as<double>());
    else
        out.push_back(as<double>());
    return out;
}

namespace yaml_detail {
inline std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r");
    return s.substr(a, b - a + 1);
}
// drop a comment: '#' at line start or after whitespace, outside quotes
inline std::string strip_comment(const std::string& s) {
    char q = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        const char c = s[i];
        if (q) {
            if (c == q) q = 0;
        } else if (c == '"' || c == '\'') {
            q = c;
        } else if (c == '#' && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t')) {
            return s.substr(0, i);
        }
    }
    return s;
}
inline YamlNode scalar(const std::string& raw) {
    YamlNode n;
    std::string v = trim(raw);
    if (v.size() >= 2 && (v[0] == '"' || v[0] == '\'') && v.back() == v[0]) v = v.substr(1, v.size() - 2);
    n.kind = YamlNode::Scalar;
    n.value = v;
    return n;
}
inline YamlNode value_of(const std::string& raw) {
    const std::string v = trim(raw);
    if (v.size() >= 2 && v[0] == '[' && v.back() == ']') {
        YamlNode n;
        n.kind = YamlNode::Seq;
        std::string body = v.substr(1, v.size() - 2);
        std::stringstream ss(body);
        std::string item;
        while (std::getline(ss, item, ','))
            if (!trim(item).empty()) n.seq.push_back(scalar(item));
        return n;
    }
    if (v.empty()) {
        YamlNode n;
        n.defined = true;
        return n;
    }
    return scalar(v);
}
struct Line {
    int indent;
    std::string text;
    int lineno;
};
// position of the "key:" separator (a ':' followed by space or end of line, outside quotes)
inline size_t key_colon(const std::string& s) {
    char q = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        const char c = s[i];
        if (q) {
            if (c == q) q = 0;
        } else if (c == '"' || c == '\'') {
            q = c;
        } else if (c == ':' && (i + 1 == s.size() || s[i + 1] == ' ' || s[i + 1] == '\t')) {
            return i;
        }
    }
    return std::string::npos;
}
inline YamlNode parse_block(const std::vector<Line>& L, size_t& i, int indent);
inline YamlNode parse_block(const std::vector<Line>& L, size_t& i, int indent) {
    YamlNode node;
    if (i >= L.size()) return node;
    const bool is_seq = L[i].text.rfind("- ", 0) == 0 || L[i].text == "-";
    node.kind = is_seq ? YamlNode::Seq : YamlNode::Map;
    while (i < L.size() && L[i].indent == indent) {
        const Line& ln = L[i];
        if (is_seq) {
            if (!(ln.text.rfind("- ", 0) == 0 || ln.text == "-"))
                throw std::logic_error("Error: YAML line " + std::to_string(ln.lineno) + ": expected '- '\n");
            node.seq.push_back(value_of(ln.text.substr(1)));
            ++i;
            continue;
        }
        const size_t c = key_colon(ln.text);
        if (c == std::string::npos)
            throw std::logic_error("Error: YAML line " + std::to_string(ln.lineno) + ": expected 'key: value'\n");
        const std::string key = scalar(ln.text.substr(0, c)).value;
        const std::string rest = trim(ln.text.substr(c + 1));
        ++i;
        if (!rest.empty()) {
            node.map.emplace_back(key, value_of(rest));
        } else if (i < L.size() && L[i].indent > indent) {
            node.map.emplace_back(key, parse_block(L, i, L[i].indent));
        } else if (i < L.size() && L[i].indent == indent && L[i].text.rfind("- ", 0) == 0) {
            node.map.emplace_back(key, parse_block(L, i, indent));  // "key:\n- a\n- b" at the same indent
        } else {
            YamlNode empty;
            empty.defined = true;
            node.map.emplace_back(key, empty);
        }
    }
    if (i < L.size() && L[i].indent > indent)
        throw std::logic_error("Error: YAML line " + std::to_string(L[i].lineno) + ": bad indentation\n");
    return node;
}
}  // namespace yaml_detail

inline YamlNode yaml_load(const std::string& text) {
    using namespace yaml_detail;
    std::vector<Line> lines;
    std::stringstream ss(text);
    std::string raw;
    int lineno = 0;
    while (std::getline(ss, raw)) {
        ++lineno;
        if (raw.find('\t') != std::string::npos && raw.find_first_not_of(" \t") != std::string::npos &&
            raw.find_first_not_of(" ") == raw.find('\t'))
            throw std::logic_error("Error: YAML line " + std::to_string(lineno) + ": tab indentation\n");
        const std::string s = strip_comment(raw);
        const std::string t = trim(s);
        if (t.empty() || t == "---" || t == "...") continue;
        lines.push_back({(int)s.find_first_not_of(' '), t, lineno});
    }
    size_t i = 0;
    if (lines.empty()) return YamlNode();
    YamlNode root = parse_block(lines, i, lines[0].indent);
    if (i != lines.size())
        throw std::logic_error("Error: YAML line " + std::to_string(lines[i].lineno) + ": bad indentation\n");
    return root;
}

inline YamlNode yaml_load_file(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::logic_error("Fatal Error: input file " + path + " was not found!\n");
    std::stringstream ss;
    ss << f.rdbuf();
    return yaml_load(ss.str());
}

/* ------------------------------------------------------------------------------------------------ */
/* ADCIRC fort.14 (AdcircFormat + the node/element maps of MeshMetaData)                            */

struct AdcircMesh {
    std::string name;
    std::vector<uint32_t> node_names;  // ascending node name (MeshMetaData's std::map order)
    std::vector<double> node_xyz;      // [3 * n_nodes]
    std::vector<uint32_t> elem_names;  // ascending element name = the reference's element IDs
    std::vector<int32_t> elem_nodes;   // [3 * n_elems], 0-based indices into node_names
    // boundary chains in get_ibtype's search order: open (tide) boundaries, then the land-boundary
    // segments in file order, then generic boundaries (typed land)
    std::vector<int32_t> seg_type;
    std::vector<int64_t> seg_offsets{0};
    std::vector<int32_t> seg_nodes;

    int64_t n_nodes() const { return (int64_t)node_names.size(); }
    int64_t n_elems() const { return (int64_t)elem_names.size(); }

    // SWE::preprocess_mesh_data inputs: Manning's n per node and the .bcis tide / flow blocks
    std::vector<double> node_manning_n;
    struct Block {
        int32_t type = DGSW_BC_TIDE;
        std::vector<int32_t> nodes;  // indices into node_names
        std::vector<double> frequency, forcing_fact, equilib_arg;
        std::vector<double> amplitude, phase;  // [constituent][node]
    };
    std::vector<Block> forcing;
    std::vector<dgsw_forcing_block> forcing_view;
    std::vector<int32_t> levee_nodes;  // .bcis levee lines: front, back node indices
    std::vector<double> levee_data;    // H_barrier, C_subcritical, C_supercritical

    dgsw_mesh view() {
        forcing_view.clear();
        for (const Block& b : forcing) {
            dgsw_forcing_block f{};
            f.type = b.type;
            f.n_nodes = (int32_t)b.nodes.size();
            f.n_constituents = (int32_t)b.frequency.size();
            f.nodes = b.nodes.data();
            f.frequency = b.frequency.data();
            f.forcing_fact = b.forcing_fact.data();
            f.equilib_arg = b.equilib_arg.data();
            f.amplitude = b.amplitude.data();
            f.phase = b.phase.data();
            forcing_view.push_back(f);
        }
        dgsw_mesh m{};
        m.node_manning_n = node_manning_n.empty() ? nullptr : node_manning_n.data();
        m.n_forcing = (int32_t)forcing_view.size();
        m.forcing = forcing_view.empty() ? nullptr : forcing_view.data();
        m.n_levee_pairs = (int32_t)(levee_nodes.size() / 2);
        m.levee_nodes = levee_nodes.empty() ? nullptr : levee_nodes.data();
        m.levee_data = levee_data.empty() ? nullptr : levee_data.data();
        m.n_nodes = n_nodes();
        m.node_xyz = node_xyz.data();
        m.n_elems = n_elems();
        m.elem_nodes = elem_nodes.data();
        m.elem_ids = elem_names.data();
        m.n_segments = (int32_t)seg_type.size();
        m.seg_type = seg_type.data();
        m.seg_offsets = seg_offsets.data();
        m.seg_nodes = seg_nodes.data();
        return m;
    }
};

/* Reads a fort.14 like AdcircFormat::AdcircFormat (adcirc_format.cpp:3-130). IBTYPE mapping as in
 * get_ibtype (:214-259): open boundaries -> tide, IBTYPE%10==0 -> land, %10==2 -> flow, 77 -> function,
 * 88 -> outflow, %10==4 -> an internal barrier (levee) chain of its front then its back nodes; island
 * segments (%10==1) are read but never matched, so they are not emitted. */
/* The part of std::istream the mesh reader uses (>> of integers and doubles across white space and line
 * ends, ignore to the end of a line, getline, the fail state) over the whole file read at once: the same
 * tokens and values (strtol / strtod, as the stream's num_get uses) at a fraction of the cost on meshes of
 * millions of elements. */
class TextIn {
  public:
    explicit TextIn(const std::string& path) {
        std::ifstream f(path, std::ios::binary);
        if (!f) {
            ok_ = false;
            return;
        }
        f.seekg(0, std::ios::end);
        buf_.resize((size_t)f.tellg());
        f.seekg(0);
        f.read(&buf_[0], (std::streamsize)buf_.size());
        buf_.push_back('\0');
        p_ = buf_.data();
        end_ = buf_.data() + buf_.size() - 1;
    }
    explicit operator bool() const { return ok_; }
    bool operator!() const { return !ok_; }
    TextIn& operator>>(long& v) {
        if (!skip_space()) return *this;
        char* e = nullptr;
        const long x = std::strtol(p_, &e, 10);
        if (e == p_) {
            ok_ = false;
            return *this;
        }
        v = x;
        p_ = e;
        return *this;
    }
    TextIn& operator>>(double& v) {
        if (!skip_space()) return *this;
        char* e = nullptr;
        const double x = std::strtod(p_, &e);
        if (e == p_) {
            ok_ = false;
            return *this;
        }
        v = x;
        p_ = e;
        return *this;
    }
    void ignore_line() {
        while (p_ < end_ && *p_ != '\n') ++p_;
        if (p_ < end_) ++p_;
    }
    bool getline(std::string& line) {
        if (!ok_ || p_ >= end_) {
            ok_ = false;
            return false;
        }
        const char* b = p_;
        while (p_ < end_ && *p_ != '\n') ++p_;
        line.assign(b, p_);
        if (p_ < end_) ++p_;
        return true;
    }

  private:
    bool skip_space() {
        if (!ok_) return false;
        while (p_ < end_ && std::isspace((unsigned char)*p_)) ++p_;
        if (p_ >= end_) ok_ = false;
        return ok_;
    }
    std::vector<char> buf_;
    const char* p_ = nullptr;
    const char* end_ = nullptr;
    bool ok_ = true;
};

inline AdcircMesh read_adcirc(const std::string& path) {
    TextIn ifs(path);
    if (!ifs) throw std::logic_error("Fatal Error: ADCIRC mesh file " + path + " was not found!\n");
    AdcircMesh M;
    auto skip_line = [&ifs]() { ifs.ignore_line(); };
    auto fail = [&path](const std::string& what) {
        throw std::logic_error("Fatal Error: ADCIRC mesh file " + path + ": " + what + "\n");
    };
    ifs.getline(M.name);
    {
        std::stringstream ss(M.name);
        ss >> M.name;  // the reference reads the first token as the name
    }
    long ne = -1, nn = -1;
    ifs >> ne >> nn;
    skip_line();
    if (!ifs || ne < 0 || nn < 0) fail("bad element/node counts");
    // node and element tables, ordered by name as MeshMetaData's maps order them
    std::vector<std::pair<uint32_t, std::array<double, 3>>> nodes;
    nodes.reserve((size_t)nn);
    for (long i = 0; i < nn; ++i) {
        long name;
        std::array<double, 3> xyz;
        ifs >> name >> xyz[0] >> xyz[1] >> xyz[2];
        skip_line();
        if (!ifs) fail("truncated node table");
        if (name < 0) throw std::logic_error("Fatal Error: in ADCIRC mesh node ID is negative!\n");
        nodes.emplace_back((uint32_t)name, xyz);
    }
    std::vector<std::pair<uint32_t, std::array<long, 3>>> elems;
    elems.reserve((size_t)ne);
    for (long i = 0; i < ne; ++i) {
        long name, nv;
        std::array<long, 3> nd;
        ifs >> name >> nv >> nd[0] >> nd[1] >> nd[2];
        skip_line();
        if (!ifs) fail("truncated element table");
        if (name < 0) throw std::logic_error("Fatal Error: in ADCIRC mesh element ID is negative!\n");
        if (nv != 3) fail("element " + std::to_string(name) + " is not a triangle");
        elems.emplace_back((uint32_t)name, nd);
    }
    auto by_name = [](const auto& a, const auto& b) { return a.first < b.first; };
    std::stable_sort(nodes.begin(), nodes.end(), by_name);
    std::stable_sort(elems.begin(), elems.end(), by_name);
    for (size_t i = 1; i < nodes.size(); ++i)
        if (nodes[i].first == nodes[i - 1].first) fail("node " + std::to_string(nodes[i].first) + " defined twice");
    for (size_t i = 1; i < elems.size(); ++i)
        if (elems[i].first == elems[i - 1].first) fail("element " + std::to_string(elems[i].first) + " defined twice");
    M.node_names.reserve(nodes.size());
    M.node_xyz.reserve(3 * nodes.size());
    for (const auto& kv : nodes) {
        M.node_names.push_back(kv.first);
        M.node_xyz.insert(M.node_xyz.end(), kv.second.begin(), kv.second.end());
    }
    std::vector<std::pair<uint32_t, std::array<double, 3>>>().swap(nodes);
    // name -> index: a direct table when the names are dense, else a binary search
    const uint32_t max_name = M.node_names.empty() ? 0 : M.node_names.back();
    std::vector<int32_t> dense;
    if ((uint64_t)max_name < 4 * (uint64_t)M.node_names.size() + 16) {
        dense.assign((size_t)max_name + 1, -1);
        for (size_t i = 0; i < M.node_names.size(); ++i) dense[M.node_names[i]] = (int32_t)i;
    }
    auto node_index = [&](long name) -> int32_t {
        if (name >= 0 && !dense.empty()) {
            if ((uint64_t)name < dense.size() && dense[(size_t)name] >= 0) return dense[(size_t)name];
        } else if (name >= 0) {
            auto it = std::lower_bound(M.node_names.begin(), M.node_names.end(), (uint32_t)name);
            if (it != M.node_names.end() && *it == (uint32_t)name) return (int32_t)(it - M.node_names.begin());
        }
        fail("unknown node " + std::to_string(name));
        return -1;
    };
    M.elem_names.reserve(elems.size());
    M.elem_nodes.reserve(3 * elems.size());
    for (const auto& kv : elems) {
        M.elem_names.push_back(kv.first);
        for (int k = 0; k < 3; ++k) M.elem_nodes.push_back(node_index(kv.second[k]));
    }
    auto add_segment = [&](int32_t type, const std::vector<long>& chain) {
        M.seg_type.push_back(type);
        for (long n : chain) M.seg_nodes.push_back(node_index(n));
        M.seg_offsets.push_back((int64_t)M.seg_nodes.size());
    };
    long nope = 0, neta = 0;
    ifs >> nope;
    skip_line();
    ifs >> neta;
    skip_line();
    if (!ifs) return M;  // no boundary section
    std::vector<std::vector<long>> open(nope);
    for (long b = 0; b < nope; ++b) {
        long n;
        ifs >> n;
        skip_line();
        open[b].resize(n);
        for (long i = 0; i < n; ++i) {
            ifs >> open[b][i];
            skip_line();
        }
    }
    for (const auto& ch : open) add_segment(DGSW_BC_TIDE, ch);
    long nbou = 0, nvel = 0;
    ifs >> nbou;
    skip_line();
    ifs >> nvel;
    skip_line();
    for (long b = 0; b < nbou && ifs; ++b) {
        long n, ibtype;
        ifs >> n >> ibtype;
        skip_line();
        std::vector<long> chain(n);
        if (ibtype % 10 == 4) {
            // internal barrier: NBVV IBCONN BARINTH BARINCFSB BARINCFSP per line (adcirc_format.cpp:89-102);
            // the barrier heights and coefficients the RKDG step uses come from the .bcis levee lines
            std::vector<long> back(n);
            for (long i = 0; i < n; ++i) {
                double h, cs, cp;
                ifs >> chain[i] >> back[i] >> h >> cs >> cp;
                skip_line();
            }
            if (!ifs) fail("truncated internal barrier segment");
            chain.insert(chain.end(), back.begin(), back.end());
            add_segment(DGSW_BC_LEVEE, chain);
            continue;
        }
        if (!(ibtype % 10 == 0 || ibtype % 10 == 1 || ibtype % 10 == 2 || ibtype == 77 || ibtype == 88))
            throw std::logic_error("Fatal Error: undefined boundary type in ADCIRC mesh: " + std::to_string(ibtype) +
                                   "!\n");
        for (long i = 0; i < n; ++i) {
            ifs >> chain[i];
            skip_line();
        }
        if (ibtype == 77)
            add_segment(DGSW_BC_FUNCTION, chain);
        else if (ibtype == 88)
            add_segment(DGSW_BC_OUTFLOW, chain);
        else if (ibtype % 10 == 0)
            add_segment(DGSW_BC_LAND, chain);
        else if (ibtype % 10 == 2)
            add_segment(DGSW_BC_FLOW, chain);
        // ibtype % 10 == 1 (island): never matched by get_ibtype
    }
    long ngen = 0, nngn = 0;
    if (ifs >> ngen) {
        skip_line();
        ifs >> nngn;
        skip_line();
        for (long b = 0; b < ngen && ifs; ++b) {
            long n;
            ifs >> n;
            skip_line();
            std::vector<long> chain(n);
            for (long i = 0; i < n; ++i) {
                ifs >> chain[i];
                skip_line();
            }
            add_segment(DGSW_BC_LAND, chain);
        }
    }
    return M;
}

/* SWE::Inputs::read_bcis (swe_inputs.cpp:211-290): tide and flow blocks, each a "btype nnodes" line, the
 * constituent count, then per constituent "frequency forcing_fact equilib_arg" and nnodes lines
 * "node_ID amplitude phase"; levee blocks, nnodes lines "front back H_barrier C_subcritical
 * C_supercritical" (levee_is_data). Other lines are skipped. A missing file gives no
 * blocks, as in the reference (its existence check is commented out); a tide or flow face without data
 * then fails in create_boundaries' "unable to find ... data". A node ID the mesh does not have can match
 * no face and is dropped. Where the reference would append a node listed twice in one constituent to the
 * same per-node lists (shifting its constituents), or index past a node missing from a constituent, this
 * reader raises an error instead. */
inline void read_bcis(const std::string& path, AdcircMesh& M) {
    std::ifstream file(path);
    if (!file) return;
    std::map<uint32_t, int32_t> index;
    for (size_t i = 0; i < M.node_names.size(); ++i) index[M.node_names[i]] = (int32_t)i;
    constexpr unsigned levee = DGSW_BC_INTERNAL + 1;
    std::string line;
    while (std::getline(file, line)) {
        std::stringstream head(line);
        unsigned btype = 0, nnodes = 0;
        head >> btype >> nnodes;
        if (btype == DGSW_BC_TIDE || btype == DGSW_BC_FLOW) {
            AdcircMesh::Block b;
            b.type = (int32_t)btype;
            unsigned ncon = 0;
            std::getline(file, line);
            std::stringstream(line) >> ncon;
            std::vector<uint32_t> ids;                                   // first-appearance order
            std::vector<std::map<uint32_t, std::pair<double, double>>> val(ncon);
            for (unsigned con = 0; con < ncon; ++con) {
                double fr = 0, ff = 0, eq = 0;
                std::getline(file, line);
                std::stringstream(line) >> fr >> ff >> eq;
                b.frequency.push_back(fr);
                b.forcing_fact.push_back(ff);
                b.equilib_arg.push_back(eq);
                for (unsigned k = 0; k < nnodes; ++k) {
                    std::getline(file, line);
                    std::stringstream st(line);
                    uint32_t id = 0;
                    double amp = 0, ph = 0;
                    st >> id >> amp >> ph;
                    if (con == 0) ids.push_back(id);
                    if (!val[con].emplace(id, std::make_pair(amp, ph)).second)
                        throw std::logic_error("Fatal Error: .bcis block lists node " + std::to_string(id) +
                                               " twice for one constituent\n");
                }
            }
            std::vector<uint32_t> kept;
            for (uint32_t id : ids) {
                auto it = index.find(id);
                if (it == index.end()) continue;
                kept.push_back(id);
                b.nodes.push_back(it->second);
            }
            b.amplitude.resize((size_t)ncon * kept.size());
            b.phase.resize((size_t)ncon * kept.size());
            for (unsigned con = 0; con < ncon; ++con)
                for (size_t j = 0; j < kept.size(); ++j) {
                    auto it = val[con].find(kept[j]);
                    if (it == val[con].end())
                        throw std::logic_error("Fatal Error: .bcis node " + std::to_string(kept[j]) +
                                               " has no data for constituent " + std::to_string(con) + "\n");
                    b.amplitude[(size_t)con * kept.size() + j] = it->second.first;
                    b.phase[(size_t)con * kept.size() + j] = it->second.second;
                }
            M.forcing.push_back(std::move(b));
        } else if (btype == levee) {
            // "front back H_barrier C_subcritical C_supercritical"; pairs of unknown nodes match no face
            for (unsigned k = 0; k < nnodes; ++k) {
                std::getline(file, line);
                std::stringstream st(line);
                uint32_t a = 0, b = 0;
                double H = 0, cs = 0, cp = 0;
                st >> a >> b >> H >> cs >> cp;
                auto ia = index.find(a), ib = index.find(b);
                if (ia == index.end() || ib == index.end()) continue;
                M.levee_nodes.push_back(ia->second);
                M.levee_nodes.push_back(ib->second);
                M.levee_data.push_back(H);
                M.levee_data.push_back(cs);
                M.levee_data.push_back(cp);
            }
        }
    }
}

/* Manning's n (swe_pre_init_data.hpp:165-182): "node_ID n" lines up to the first that does not parse;
 * a node the file does not list gets n = 0 (the reference's std::map default). */
inline void read_manning(const std::string& path, AdcircMesh& M) {
    std::ifstream file(path);
    if (!file)
        throw std::logic_error("Fatal Error: manning factor data file " + path + " was not found!\n");
    std::map<uint32_t, int32_t> index;
    for (size_t i = 0; i < M.node_names.size(); ++i) index[M.node_names[i]] = (int32_t)i;
    M.node_manning_n.assign(M.node_names.size(), 0.0);
    std::string line;
    while (std::getline(file, line)) {
        std::istringstream st(line);
        uint32_t id;
        double n;
        if (!(st >> id >> n)) break;
        auto it = index.find(id);
        if (it != index.end()) M.node_manning_n[it->second] = n;
    }
}

/* a path from the input file, relative to the input file's directory unless absolute */
inline std::string input_relative(const std::string& dir, const std::string& path) {
    return (!path.empty() && path[0] == '/') ? path : dir + path;
}

/* ------------------------------------------------------------------------------------------------ */
/* input parameters                                                                                 */

/* SWE::Inputs (swe_inputs.hpp:125-158) restricted to what the RKDG step reads; defaults as there */
struct SWEInputs {
    std::string name;
    double g = 9.81;
    double rho_air = 1.2250;
    double rho_water = 1000.0;
    bool spherical = false;
    double longitude_o = 0.0, latitude_o = 0.0, R = 6378200.0;
    int ic_type = 0;  // 0 Default/Constant, 1 Function
    double ze_initial = 0.0, qx_initial = 0.0, qy_initial = 0.0;
    bool function_source = false;
    bool wetting_drying = false;
    double h_o = 0.1;
    bool slope_limiting = false;
    double sl_M = 1.0e-8, sl_nu = 1.5;
    int bottom_friction = DGSW_FRICTION_NONE;  // BottomFrictionType None / Chezy / Manning
    double friction_coefficient = 0.0;
    std::string manning_data_file;

    SWEInputs() = default;
    /* SWE::Inputs::Inputs (swe_inputs.cpp:4-205): malformed optional nodes warn and keep defaults */
    explicit SWEInputs(const YamlNode& n) {
        if (!n["name"]) throw std::logic_error("Error: problem name not specified\n");
        name = n["name"].as<std::string>();
        if (n["gravity"]) g = n["gravity"].as<double>();
        if (n["density_air"]) rho_air = n["density_air"].as<double>();
        if (n["density_water"]) rho_water = n["density_water"].as<double>();
        if (const YamlNode& sp = n["spherical_projection"]) {
            if (sp["longitude_o"] && sp["latitude_o"] && sp["R"]) {
                spherical = true;
                longitude_o = sp["longitude_o"].as<double>();
                latitude_o = sp["latitude_o"].as<double>();
                R = sp["R"].as<double>();
            } else {
                std::cerr << "Warning: spherical projection inputs are mal-formatted. Using default parameters.\n";
            }
        }
        if (const YamlNode& ic = n["initial_conditions"]) {
            const std::string w = "Warning: initial conditions are mal-formatted. Using default parameters.\n";
            if (ic["type"]) {
                const std::string t = ic["type"].as<std::string>();
                if (t == "Constant") {
                    if (ic["initial_surface_height"] && ic["initial_momentum_x"] && ic["initial_momentum_y"]) {
                        ic_type = 0;
                        ze_initial = ic["initial_surface_height"].as<double>();
                        qx_initial = ic["initial_momentum_x"].as<double>();
                        qy_initial = ic["initial_momentum_y"].as<double>();
                    } else {
                        std::cerr << w;
                    }
                } else if (t == "Function") {
                    ic_type = 1;
                } else {
                    std::cerr << w;
                }
            } else {
                std::cerr << w;
            }
        }
        if (const YamlNode& fs = n["function_source"]) {
            if (!fs.IsNull() && fs.as<std::string>() == "Enable")
                function_source = true;
            else
                std::cerr << "Warning: function source is mal-formatted. Using default parameters.\n";
        }
        if (const YamlNode& bf = n["bottom_friction"]) {  // swe_inputs.cpp:86-123
            const std::string w = "Warning: bottom friction is mal-formatted. Using default parameters.\n";
            const std::string t = bf["type"] ? bf["type"].as<std::string>() : std::string();
            if (t == "Chezy" && bf["coefficient"]) {
                bottom_friction = DGSW_FRICTION_CHEZY;
                friction_coefficient = bf["coefficient"].as<double>();
            } else if (t == "Manning" && bf["coefficient"] && bf["input_file"]) {
                bottom_friction = DGSW_FRICTION_MANNING;
                friction_coefficient = bf["coefficient"].as<double>();
                manning_data_file = bf["input_file"].as<std::string>();
            } else {
                std::cerr << w;
            }
            if (bottom_friction != DGSW_FRICTION_NONE && friction_coefficient < 0.)
                throw std::logic_error("Fatal Error: Chezy friction coefficient must be postive!\n");
        }
        if (n["meteo_forcing"] && n["meteo_forcing"]["type"])
            throw Error(DGSW_ERR_UNSUPPORTED, "meteo forcing is not supported by this build");
        if (n["tide_potential"] && n["tide_potential"]["type"])
            throw Error(DGSW_ERR_UNSUPPORTED, "tide potential forcing is not supported by this build");
        if (const YamlNode& co = n["coriolis"])
            if (!co.IsNull() && co.as<std::string>() == "Enable")
                throw Error(DGSW_ERR_UNSUPPORTED, "Coriolis forcing is not supported by this build");
        if (const YamlNode& wd = n["wetting_drying"]) {
            if (wd["h_o"]) {
                wetting_drying = true;
                h_o = wd["h_o"].as<double>();
            } else {
                std::cerr << "Warning: wet-dry is mal-formatted. Using default parameters.\n";
            }
        }
        if (const YamlNode& sl = n["slope_limiting"]) {
            const std::string w = "Warning: slope limiting is mal-formatted. Using default parameters.\n";
            if (sl["type"] && sl["type"].as<std::string>() == "Cockburn-Shu" && sl["M"] && sl["nu"]) {
                slope_limiting = true;
                sl_M = sl["M"].as<double>();
                sl_nu = sl["nu"].as<double>();
            } else {
                std::cerr << w;
            }
        }
    }
};

/* the `b200:` extension node (see the file comment) */
struct B200Input {
    int function_set = 0;
    std::vector<double> function_parameters;
    int precision = DGSW_FP64;
    int tile = 0;
    int device = 0;

    B200Input() = default;
    explicit B200Input(const YamlNode& n) {
        if (!n) return;
        if (const YamlNode& fs = n["function_set"]) {
            static const char* names[] = {"none", "reference_manufactured", "manufactured_sine", "thacker_bowl",
                                          "gaussian_humps"};
            const std::string s = fs.as<std::string>();
            function_set = -1;
            for (int i = 0; i < 5; ++i)
                if (s == names[i]) function_set = i;
            if (function_set < 0) throw std::logic_error("Error: unknown b200.function_set: " + s + "\n");
        }
        if (n["function_parameters"]) function_parameters = n["function_parameters"].as<std::vector<double>>();
        if (function_parameters.size() > 16) throw std::logic_error("Error: more than 16 b200.function_parameters\n");
        if (const YamlNode& p = n["precision"]) {
            const std::string s = p.as<std::string>();
            if (s == "fp64")
                precision = DGSW_FP64;
            else if (s == "fp32")
                precision = DGSW_FP32;
            else
                throw std::logic_error("Error: b200.precision must be fp64 or fp32\n");
        }
        if (n["tile"]) tile = n["tile"].as<int>();
        if (n["device"]) device = n["device"].as<int>();
    }
};

struct MeshInput {
    std::string mesh_format, mesh_file_name, bc_is_file_name, coordinate_system;
};

struct StepperInput {
    double run_time = 0.0, dt = 0.0, ramp_duration = 0.0;
    unsigned nstages = 0, order = 0;
};

struct WriterInput {
    bool writing_output = false;
    std::string output_path;
    bool writing_vtk_output = false;
    double vtk_output_frequency = 0.0;
    unsigned vtk_output_freq_step = 0;
    bool writing_vtu_output = false;
    double vtu_output_frequency = 0.0;
    unsigned vtu_output_freq_step = 0;
    bool writing_modal_output = false;
    double modal_output_frequency = 0.0;
    unsigned modal_output_freq_step = 0;
};

/* InputParameters<SWE::Inputs> (input_parameters.hpp:95-261) */
struct InputParameters {
    unsigned polynomial_order = 0;
    MeshInput mesh_input;
    StepperInput stepper_input;
    SWEInputs problem_input;
    WriterInput writer_input;
    B200Input b200;
    std::string input_dir;  // mesh paths are relative to the input file's directory

    InputParameters() = default;
    explicit InputParameters(const std::string& input_path) {
        const YamlNode f = yaml_load_file(input_path);
        const size_t slash = input_path.find_last_of('/');
        input_dir = slash == std::string::npos ? "" : input_path.substr(0, slash + 1);
        if (!f["polynomial_order"]) throw std::logic_error("Error: P YAML node not specified\n");
        polynomial_order = f["polynomial_order"].as<unsigned>();
        const YamlNode& mesh = f["mesh"];
        if (!mesh) throw std::logic_error("Error: Mesh YAML node not specified\n");
        if (!(mesh["format"] && mesh["file_name"] && mesh["coordinate_system"]))
            throw std::logic_error("Error: Mesh YAML node is malformatted\n");
        mesh_input.mesh_format = mesh["format"].as<std::string>();
        if (mesh_input.mesh_format != "Adcirc")
            throw std::logic_error("Error: Unsupported mesh format: " + mesh_input.mesh_format + '\n');
        mesh_input.mesh_file_name = mesh["file_name"].as<std::string>();
        mesh_input.bc_is_file_name =
            mesh_input.mesh_file_name.substr(0, mesh_input.mesh_file_name.find_last_of('.')) + ".bcis";
        mesh_input.coordinate_system = mesh["coordinate_system"].as<std::string>();
        if (mesh_input.coordinate_system != "cartesian" && mesh_input.coordinate_system != "polar" &&
            mesh_input.coordinate_system != "spherical")
            throw std::logic_error("Error: Unsupported coordinate system: " + mesh_input.coordinate_system + '\n');
        const YamlNode& ts = f["timestepping"];
        if (!ts) throw std::logic_error("Error: Timestepping YAML node not specified\n");
        if (!(ts["start_time"] && ts["end_time"] && ts["dt"] && ts["order"] && ts["nstages"]))
            throw std::logic_error("Error: Timestepping YAML node is malformatted\n");
        stepper_input.run_time = parse_time(ts["end_time"].as<std::string>()) -
                                 parse_time(ts["start_time"].as<std::string>());
        stepper_input.dt = ts["dt"].as<double>();
        stepper_input.order = ts["order"].as<unsigned>();
        stepper_input.nstages = ts["nstages"].as<unsigned>();
        stepper_input.ramp_duration = ts["ramp_duration"] ? ts["ramp_duration"].as<double>() : 0.0;
        const YamlNode& prob = f["problem"];
        if (!prob) throw std::logic_error("Error: Problem YAML node not specified\n");
        problem_input = SWEInputs(prob);
        if (problem_input.name != "rkdg_swe")
            throw Error(DGSW_ERR_UNSUPPORTED, "problem " + problem_input.name + " is not rkdg_swe");
        if (const YamlNode& out = f["output"]) {
            if (!out["path"]) throw std::logic_error("Error: Output YAML node is malformatted\n");
            writer_input.writing_output = true;
            writer_input.output_path = out["path"].as<std::string>();
            if (writer_input.output_path.empty() || writer_input.output_path.back() != '/')
                writer_input.output_path += "/";
            if (const YamlNode& vk = out["vtk"]) {
                if (!vk["frequency"]) throw std::logic_error("Error: VTK YAML node is malformatted\n");
                writer_input.writing_vtk_output = true;
                writer_input.vtk_output_frequency = vk["frequency"].as<double>();
                writer_input.vtk_output_freq_step =
                    (unsigned)std::ceil(writer_input.vtk_output_frequency / stepper_input.dt);
            }
            if (const YamlNode& vu = out["vtu"]) {
                if (!vu["frequency"]) throw std::logic_error("Error: VTU YAML node is malformatted\n");
                writer_input.writing_vtu_output = true;
                writer_input.vtu_output_frequency = vu["frequency"].as<double>();
                writer_input.vtu_output_freq_step =
                    (unsigned)std::ceil(writer_input.vtu_output_frequency / stepper_input.dt);
            }
            if (const YamlNode& mo = out["modal"]) {
                if (!mo["frequency"]) throw std::logic_error("Error: Modal YAML node is malformatted\n");
                writer_input.writing_modal_output = true;
                writer_input.modal_output_frequency = mo["frequency"].as<double>();
                writer_input.modal_output_freq_step =
                    (unsigned)std::ceil(writer_input.modal_output_frequency / stepper_input.dt);
            }
        }
        b200 = B200Input(f["b200"]);
    }

    /* "%d-%m-%Y %H:%M:%S" read with strptime and converted with timegm, as the reference does; a
     * missing seconds field leaves the remaining fields zero */
    static double parse_time(const std::string& s) {
        struct tm t = {};
        strptime(s.c_str(), "%d-%m-%Y %H:%M:%S", &t);
        return (double)timegm(&t);
    }
};

/* ------------------------------------------------------------------------------------------------ */
/* handle, stepper and discretization                                                               */

/* owns one library handle */
class Handle {
  public:
    Handle() = default;
    Handle(const dgsw_config& cfg, const dgsw_mesh& mesh) {
        check(dgsw_rkdg_create(&cfg, &mesh, &h_), "dgsw_rkdg_create");
    }
    ~Handle() {
        if (h_) dgsw_rkdg_destroy(h_);
    }
    Handle(const Handle&) = delete;
    Handle& operator=(const Handle&) = delete;
    Handle(Handle&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
    Handle& operator=(Handle&& o) noexcept {
        std::swap(h_, o.h_);
        return *this;
    }
    dgsw_handle get() const { return h_; }
    explicit operator bool() const { return h_ != nullptr; }

  private:
    dgsw_handle h_ = nullptr;
};

/* ESSPRKStepper's queries (explicit_ssp_rk_stepper.hpp:36-65); the state lives in the library */
class GpuStepper {
  public:
    GpuStepper() = default;
    explicit GpuStepper(const StepperInput& in) : in_(in) {}
    void bind(dgsw_handle h) { h_ = h; }
    unsigned GetOrder() const { return in_.order; }
    unsigned GetNumStages() const { return in_.nstages; }
    double GetDT() const { return in_.dt; }
    double GetRampDuration() const { return in_.ramp_duration; }
    double GetTimeAtCurrentStage() const { return query().t; }
    uint64_t GetStep() const { return (uint64_t)query().step; }
    unsigned GetStage() const { return (unsigned)query().stage; }

  private:
    struct Q {
        double t;
        int64_t step;
        int32_t stage;
    };
    Q query() const {
        Q q{0.0, 0, 0};
        if (h_) check(dgsw_rkdg_get_time(h_, &q.t, &q.step, &q.stage), "dgsw_rkdg_get_time");
        return q;
    }
    StepperInput in_;
    dgsw_handle h_ = nullptr;
};

/* SWE::preprocess_mesh_data (swe_pre_preprocess_mesh.hpp:6-27): a mesh in spherical coordinates
 * (longitude, latitude in degrees) is projected onto the cylinder through (longitude_o, latitude_o),
 * with the reference's PI = 3.14159265359 */
inline void project_spherical(const InputParameters& input, AdcircMesh& mesh) {
    if (input.mesh_input.coordinate_system != "spherical") return;
    const SWEInputs& pi = input.problem_input;
    if (!pi.spherical) {
        std::cerr << "Warning: Spherical projection input not provided! Using default values to perfrom projection!\n";
        std::cerr << "Consider using spherical projection to account for geometric distortion!\n";
    }
    constexpr double PI = 3.14159265359;
    const double R_o = pi.R * std::cos(pi.latitude_o * PI / 180.0);
    for (size_t n = 0; n < mesh.node_names.size(); ++n) {
        mesh.node_xyz[3 * n] = R_o * (mesh.node_xyz[3 * n] - pi.longitude_o) * PI / 180.0;
        mesh.node_xyz[3 * n + 1] = pi.R * mesh.node_xyz[3 * n + 1] * PI / 180.0;
    }
}

/* DGDiscretization<Problem>: the mesh plus the library handle that holds all element data */
struct GpuDiscretization {
    AdcircMesh mesh;
    dgsw_config config;
    Handle handle;

    void initialize(const InputParameters& input) {
        mesh = read_adcirc(input_relative(input.input_dir, input.mesh_input.mesh_file_name));
        project_spherical(input, mesh);
        // Simulation ctor: input.read_bcis(); initialize_data_serial: the Manning n file
        read_bcis(input_relative(input.input_dir, input.mesh_input.bc_is_file_name), mesh);
        if (input.problem_input.bottom_friction == DGSW_FRICTION_MANNING)
            read_manning(input_relative(input.input_dir, input.problem_input.manning_data_file), mesh);
        dgsw_config_default(&config);
        const SWEInputs& pi = input.problem_input;
        config.p = (int32_t)input.polynomial_order;
        config.rk_nstages = (int32_t)input.stepper_input.nstages;
        config.rk_order = (int32_t)input.stepper_input.order;
        config.dt = input.stepper_input.dt;
        config.g = pi.g;
        config.wetting_drying = pi.wetting_drying;
        config.h_o = pi.h_o;
        config.slope_limiting = pi.slope_limiting;
        config.sl_M = pi.sl_M;
        config.sl_nu = pi.sl_nu;
        config.function_source = pi.function_source;
        config.ic_type = pi.ic_type;
        config.ic_const[0] = pi.ze_initial;
        config.ic_const[1] = pi.qx_initial;
        config.ic_const[2] = pi.qy_initial;
        config.function_set = input.b200.function_set;
        for (size_t i = 0; i < input.b200.function_parameters.size(); ++i)
            config.fn_params[i] = input.b200.function_parameters[i];
        config.spherical = pi.spherical;
        config.sp_lat0_deg = pi.latitude_o;
        config.sp_R = pi.R;
        config.bottom_friction = pi.bottom_friction;
        config.friction_cf = pi.friction_coefficient;
        config.ramp_duration = input.stepper_input.ramp_duration;
        config.precision = input.b200.precision;
        config.device = input.b200.device;
        config.tile = input.b200.tile;
        const dgsw_mesh m = mesh.view();
        handle = Handle(config, m);
    }
};

struct GpuGlobalData {};  // SWE::GlobalData holds nothing the serial RKDG step needs

/* Writer (source/simulation/writer.hpp:100-193) with the SWE writers of problem_postprocessor/:
 * modal (swe_post_write_modal.hpp:6-88), VTK (swe_post_write_vtk.hpp:5-95) and VTU
 * (swe_post_write_vtu.hpp:5-104) at the reference's N_DIV = 1 (one cell per element, its three vertices as
 * points). Field values are evaluated on the device (dgsw_rkdg_postprocess); the text formats, file names
 * and cadence (step 0 through WriteFirstStep, then every freq_step steps) are the reference's. */
class GpuWriter {
  public:
    GpuWriter() = default;
    explicit GpuWriter(const WriterInput& in) : in_(in) {}
    bool WritingOutput() const { return in_.writing_output; }
    bool WritingModalOutput() const { return in_.writing_modal_output; }

    void WriteFirstStep(const GpuDiscretization& d, const GpuStepper& stepper) { WriteOutput(d, stepper); }

    void WriteOutput(const GpuDiscretization& d, const GpuStepper& stepper) {
        const uint64_t step = (uint64_t)stepper.GetStep();
        const bool vtk = in_.writing_vtk_output && in_.vtk_output_freq_step && step % in_.vtk_output_freq_step == 0;
        const bool vtu = in_.writing_vtu_output && in_.vtu_output_freq_step && step % in_.vtu_output_freq_step == 0;
        if (vtk || vtu) {
            Fields F = fields(d);
            if (vtk) WriteVTK(d, F, step);
            if (vtu) WriteVTU(d, F, step);
        }
        if (in_.writing_modal_output && in_.modal_output_freq_step && step % in_.modal_output_freq_step == 0)
            WriteModal(d, stepper);
    }

    /* write_modal_data: <mesh>_modal_{ze,qx,qy,bath}.txt, a time line (std::to_string) and one
     * "ID value" line per element and mode; truncated at step 0, appended afterwards */
    void WriteModal(const GpuDiscretization& d, const GpuStepper& stepper) {
        dgsw_info info;
        check(dgsw_rkdg_info(d.handle.get(), &info), "dgsw_rkdg_info");
        const int nd = info.ndof;
        std::vector<double> q((size_t)info.n_elems * 3 * nd), b((size_t)info.n_elems * nd);
        check(dgsw_rkdg_get_state(d.handle.get(), q.data()), "dgsw_rkdg_get_state");
        check(dgsw_rkdg_get_bathymetry(d.handle.get(), b.data()), "dgsw_rkdg_get_bathymetry");
        const char* names[4] = {"ze", "qx", "qy", "bath"};
        for (int v = 0; v < 4; ++v) {
            const std::string name = in_.output_path + d.mesh.name + "_modal_" + names[v] + ".txt";
            std::ofstream f(name, stepper.GetStep() == 0 ? std::ios::trunc : std::ios::app);
            f << std::to_string(stepper.GetTimeAtCurrentStage()) << std::endl;
            for (int64_t e = 0; e < info.n_elems; ++e)
                for (int k = 0; k < nd; ++k)
                    f << d.mesh.elem_names[e] << ' ' << std::scientific
                      << (v < 3 ? q[((size_t)e * 3 + v) * nd + k] : b[(size_t)e * nd + k]) << std::endl;
        }
    }

    void Tick(const GpuDiscretization& d, const GpuStepper& stepper) { WriteOutput(d, stepper); }

  private:
    struct Fields {
        std::vector<double> point, cell;  // [ne][3][4], [ne][4]: ze, qx, qy, bath
        std::vector<uint8_t> wet, went_dry;
    };

    static Fields fields(const GpuDiscretization& d) {
        const int64_t ne = d.mesh.n_elems();
        Fields F;
        F.point.resize((size_t)ne * 12);
        F.cell.resize((size_t)ne * 4);
        F.wet.resize((size_t)ne);
        F.went_dry.resize((size_t)ne);
        check(dgsw_rkdg_postprocess(d.handle.get(), F.point.data(), F.cell.data(), F.wet.data(), F.went_dry.data()),
              "dgsw_rkdg_postprocess");
        return F;
    }

    /* InitializeMeshGeometryVTK + write_VTK_data, merged into <mesh>_data_<step>.vtk */
    void WriteVTK(const GpuDiscretization& d, const Fields& F, uint64_t step) {
        const AdcircMesh& M = d.mesh;
        const int64_t ne = M.n_elems();
        std::ofstream f(in_.output_path + M.name + "_data_" + std::to_string(step) + ".vtk", std::ios::binary);
        f << "# vtk DataFile Version 3.0\n";
        f << "OUTPUT DATA\n";
        f << "ASCII\n";
        f << "DATASET UNSTRUCTURED_GRID\n";
        f << "POINTS " << 3 * ne << " double\n";
        for (int64_t e = 0; e < ne; ++e)
            for (int k = 0; k < 3; ++k) {
                const int32_t n = M.elem_nodes[3 * e + k];
                f << M.node_xyz[3 * n] << '\t' << M.node_xyz[3 * n + 1] << '\t' << 0.0 << '\n';
            }
        f << "CELLS " << ne << ' ' << 4 * ne << '\n';
        for (int64_t e = 0; e < ne; ++e) f << 3 << '\t' << 3 * e << '\t' << 3 * e + 1 << '\t' << 3 * e + 2 << '\t' << '\n';
        f << "CELL_TYPES " << ne << '\n';
        for (int64_t e = 0; e < ne; ++e) f << 5 << '\n';
        f << "CELL_DATA " << ne << std::endl;
        const char* cn[4] = {"ze_cell", "qx_cell", "qy_cell", "bath_cell"};
        for (int c = 0; c < 4; ++c) {
            f << "SCALARS " << cn[c] << " double 1" << std::endl << "LOOKUP_TABLE default" << std::endl;
            for (int64_t e = 0; e < ne; ++e) f << (float)F.cell[(size_t)e * 4 + c] << std::endl;
        }
        f << "SCALARS ID unsigned_int 1" << std::endl << "LOOKUP_TABLE default" << std::endl;
        for (int64_t e = 0; e < ne; ++e) f << M.elem_names[e] << std::endl;
        f << "SCALARS wet_dry bit 1" << std::endl << "LOOKUP_TABLE default" << std::endl;
        for (int64_t e = 0; e < ne; ++e) f << (F.wet[e] != 0) << std::endl;
        f << "SCALARS went_completely_dry bit 1" << std::endl << "LOOKUP_TABLE default" << std::endl;
        for (int64_t e = 0; e < ne; ++e) f << (F.went_dry[e] != 0) << std::endl;
        f << "POINT_DATA " << 3 * ne << std::endl;
        const char* pn[4] = {"ze_point", "qx_point", "qy_point", "bath_point"};
        for (int c = 0; c < 4; ++c) {
            f << "SCALARS " << pn[c] << " double 1" << std::endl << "LOOKUP_TABLE default" << std::endl;
            for (size_t i = 0; i < (size_t)ne * 3; ++i) f << (float)F.point[i * 4 + c] << std::endl;
        }
    }

    /* InitializeMeshGeometryVTU (head, foot) + write_VTU_data, merged into <mesh>_data_<step>.vtu */
    void WriteVTU(const GpuDiscretization& d, const Fields& F, uint64_t step) {
        const AdcircMesh& M = d.mesh;
        const int64_t ne = M.n_elems();
        std::ofstream f(in_.output_path + M.name + "_data_" + std::to_string(step) + ".vtu", std::ios::binary);
        f << "<?xml version=\"1.0\"?>\n";
        f << "<VTKFile type=\"UnstructuredGrid\">\n";
        f << "\t<UnstructuredGrid>\n";
        f << "\t\t<Piece NumberOfPoints=\"" << 3 * ne << "\" NumberOfCells=\"" << ne << "\">\n";
        auto open = [&](const char* type, const char* name) {
            f << "\t\t\t\t<DataArray type=\"" << type << "\" Name=\"" << name << "\" format=\"ascii\">\n\t\t\t\t\t";
        };
        auto close = [&]() { f << "\n\t\t\t\t</DataArray>\n"; };
        f << "\t\t\t<PointData>\n";
        const char* pn[4] = {"ze_point", "qx_point", "qy_point", "bath_point"};
        for (int c = 0; c < 4; ++c) {
            open("Float32", pn[c]);
            for (size_t i = 0; i < (size_t)ne * 3; ++i) f << (float)F.point[i * 4 + c] << ' ';
            close();
        }
        open("Float32", "velocity_point");
        for (size_t i = 0; i < (size_t)ne * 3; ++i) {
            const double* v = &F.point[i * 4];
            f << (float)(std::hypot(v[1], v[2]) / (v[0] + v[3])) << ' ';
        }
        close();
        f << "\t\t\t</PointData>\n";
        f << "\t\t\t<CellData>\n";
        const char* cn[4] = {"ze_cell", "qx_cell", "qy_cell", "bath_cell"};
        for (int c = 0; c < 4; ++c) {
            open("Float32", cn[c]);
            for (int64_t e = 0; e < ne; ++e) f << (float)F.cell[(size_t)e * 4 + c] << ' ';
            close();
        }
        open("UInt32", "ID");
        for (int64_t e = 0; e < ne; ++e) f << M.elem_names[e] << ' ';
        close();
        open("Int8", "wet_dry");
        for (int64_t e = 0; e < ne; ++e) f << (F.wet[e] != 0) << ' ';
        close();
        open("Int8", "went_completely_dry");
        for (int64_t e = 0; e < ne; ++e) f << (F.went_dry[e] != 0) << ' ';
        close();
        f << "\t\t\t</CellData>\n";
        f << "\t\t\t<Points>\n";
        f << "\t\t\t\t<DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n\t\t\t\t\t";
        for (int64_t e = 0; e < ne; ++e)
            for (int k = 0; k < 3; ++k) {
                const int32_t n = M.elem_nodes[3 * e + k];
                f << M.node_xyz[3 * n] << ' ' << M.node_xyz[3 * n + 1] << ' ' << 0.0 << ' ';
            }
        f << "\n\t\t\t\t</DataArray>\n";
        f << "\t\t\t</Points>\n";
        f << "\t\t\t<Cells>\n";
        f << "\t\t\t\t<DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n\t\t\t\t\t";
        for (int64_t e = 0; e < ne; ++e) f << 3 * e << ' ' << 3 * e + 1 << ' ' << 3 * e + 2 << ' ';
        f << "\n\t\t\t\t</DataArray>\n";
        f << "\t\t\t\t<DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n\t\t\t\t\t";
        for (int64_t e = 0; e < ne; ++e) f << 3 * (e + 1) << ' ';
        f << "\n\t\t\t\t</DataArray>\n";
        f << "\t\t\t\t<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n\t\t\t\t\t";
        for (int64_t e = 0; e < ne; ++e) f << 5 << ' ';
        f << "\n\t\t\t\t</DataArray>\n";
        f << "\t\t\t</Cells>\n";
        f << "\t\t</Piece>\n";
        f << "\t</UnstructuredGrid>\n";
        f << "</VTKFile>\n";
    }

    WriterInput in_;
};

}  // namespace dgsw

/* ------------------------------------------------------------------------------------------------ */
/* the problem type                                                                                 */

namespace SWE {
namespace RKDG {

/* SWE::RKDG::Problem (rkdg_swe_problem.hpp:34-194) with the element/interface/boundary kernels fused
 * into the library's stage kernel: volume_kernel, source_kernel, interface_kernel and boundary_kernel
 * have no separate entry points, stage_serial runs all of them for every element at once. */
struct GpuProblem {
    using ProblemInputType = dgsw::SWEInputs;
    using ProblemStepperType = dgsw::GpuStepper;
    using ProblemWriterType = dgsw::GpuWriter;
    using ProblemGlobalDataType = dgsw::GpuGlobalData;
    using ProblemDiscretizationType = dgsw::GpuDiscretization;
    using ProblemInputParametersType = dgsw::InputParameters;

    /* SWE::initialize_problem_parameters: g, densities and the spherical projection are carried in the
     * handle's configuration instead of process-wide statics */
    static void initialize_problem_parameters(const ProblemInputType&) {}

    /* SWE::preprocess_mesh_data: the node projection of spherical meshes, the .bcis tide / flow / levee
     * data and the Manning n file are applied / read when the discretization is initialised
     * (GpuDiscretization::initialize) */
    static void preprocess_mesh_data(ProblemInputParametersType&) {}

    /* swe_pre_serial.hpp: initial projections, wet/dry and limiter initialisation on the device */
    static void preprocessor_serial(ProblemDiscretizationType& d, ProblemGlobalDataType&, ProblemStepperType& stepper,
                                    const ProblemInputType&) {
        stepper.bind(d.handle.get());
        dgsw::check(dgsw_rkdg_init_state(d.handle.get()), "dgsw_rkdg_init_state");
    }

    /* rkdg_swe_proc_serial_step.hpp:10-27: all stages of one step */
    static void step_serial(ProblemDiscretizationType& d, ProblemGlobalDataType&, ProblemStepperType& stepper,
                            ProblemWriterType& writer) {
        dgsw::check(dgsw_rkdg_step(d.handle.get(), 1), "dgsw_rkdg_step");
        writer.Tick(d, stepper);
    }

    /* rkdg_swe_proc_serial_step.hpp:29-67: one stage (a NaN raises dgsw::Error with DGSW_ERR_NAN where the
     * reference aborts) */
    static void stage_serial(ProblemDiscretizationType& d, ProblemGlobalDataType&, ProblemStepperType&) {
        dgsw::check(dgsw_rkdg_stage(d.handle.get()), "dgsw_rkdg_stage");
    }

    /* swe_post_comp_res_l2.hpp:7-14 summed over all elements (the square of the L2 error) */
    static double compute_residual_L2(const ProblemStepperType&, const ProblemDiscretizationType& d) {
        double l2 = 0.0;
        dgsw::check(dgsw_rkdg_l2_error(d.handle.get(), &l2), "dgsw_rkdg_l2_error");
        return l2 * l2;
    }

    static void finalize_simulation(ProblemGlobalDataType&) {}
};

}  // namespace RKDG
}  // namespace SWE

namespace Serial {

/* Serial::Simulation<ProblemType> (simulation.hpp:14-93) */
template <typename ProblemType>
class GpuSimulation {
  public:
    explicit GpuSimulation(const std::string& input_path) : input_(input_path) {
        ProblemType::initialize_problem_parameters(input_.problem_input);
        ProblemType::preprocess_mesh_data(input_);
        n_steps_ = (uint64_t)std::ceil(input_.stepper_input.run_time / input_.stepper_input.dt);
        stepper_ = typename ProblemType::ProblemStepperType(input_.stepper_input);
        writer_ = typename ProblemType::ProblemWriterType(input_.writer_input);
        discretization_.initialize(input_);
    }

    void Run() {
        ProblemType::preprocessor_serial(discretization_, global_data_, stepper_, input_.problem_input);
        if (writer_.WritingOutput()) writer_.WriteFirstStep(discretization_, stepper_);
        for (uint64_t step = 1; step <= n_steps_; ++step)
            ProblemType::step_serial(discretization_, global_data_, stepper_, writer_);
    }

    /* prints "L2 error: " with 15 digits, as the reference does */
    double ComputeL2Residual() {
        const double r = std::sqrt(ProblemType::compute_residual_L2(stepper_, discretization_));
        std::cout << "L2 error: " << std::setprecision(15) << r << std::endl;
        return r;
    }

    void Finalize() { ProblemType::finalize_simulation(global_data_); }

    uint64_t n_steps() const { return n_steps_; }
    const dgsw::InputParameters& input() const { return input_; }
    typename ProblemType::ProblemDiscretizationType& discretization() { return discretization_; }
    typename ProblemType::ProblemStepperType& stepper() { return stepper_; }

  private:
    dgsw::InputParameters input_;
    uint64_t n_steps_ = 0;
    typename ProblemType::ProblemDiscretizationType discretization_;
    typename ProblemType::ProblemGlobalDataType global_data_;
    typename ProblemType::ProblemStepperType stepper_;
    typename ProblemType::ProblemWriterType writer_;
};

}  // namespace Serial

#endif /* DGSW_RKDG_PROBLEM_HPP */
