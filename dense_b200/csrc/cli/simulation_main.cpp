// dense_simulation_<model>: DENSE's deterministic `simulation` command,
// running on the B200 engine through the C ABI of include/dense_b200.h.
//
// Same flags (arg_parse.hpp:47-96, parse_static_args arg_parse.hpp:98-171):
//   -p/--param-sets <csv>  -t/--time-total <min>  -u/--anlys-intvl <min>
//   -s/--step-size <min>  -c/--cell-total <n> -w/--tissue-width <n> |
//   -f/--cell-graph <file>  -d/--initial-conc <csv>  -a/--analysis <xml>
//   -e/--data-export <csv>  -o/--specie-option <list>  -v/--time-col
//   -i/--data-import <csv>  -N/--test-run  -n/--no-color  -h/--help
// plus --precision fp64|fp32 (FP32 rates with Kahan-compensated state) and
// --device <ordinal>.
//
// Outputs follow DENSE: each analysis of analyses.xml writes its show() text
// to its <out-file> (stdout when empty), one file per parameter set named
// x_####.y when there are several sets (run_simulation.hpp:54-63, 113-121);
// -e writes csvw_sim's trajectory export; without -a and -e a Basic analysis
// of every species and cell goes to stdout unless -N.
//
// Inputs DENSE reads out of bounds are refused or documented here: an
// analysis whose cell range leaves the tissue is skipped with a warning
// (DENSE reads past its arrays for it), and -b takes one global factor or a
// per-reaction CSV whose factors only enter the history sizing (DENSE's own
// -b reads NUM_PARAMS factors from a NUM_REACTIONS array).

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "dense_b200.h"

namespace {

// ------------------------------------------------------------------ flags
struct Args {
  std::vector<std::string> v;
  int index(const char* s, const char* l, bool next) const {
    const std::string a = std::string("-") + s, b = std::string("--") + l;
    for (size_t i = 0; i < v.size(); ++i)
      if (v[i] == a || v[i] == b) {
        if (!next) return static_cast<int>(i);
        if (i + 1 < v.size()) return static_cast<int>(i + 1);
        std::cout << "Command line argument search failed. No argument provided after flag [" << a << " | " << b
                  << "].\n";
        return -1;
      }
    return -1;
  }
  bool has(const char* s, const char* l) const { return index(s, l, false) >= 0; }
  bool str(const char* s, const char* l, std::string* out) const {
    int i = index(s, l, true);
    if (i < 0) return false;
    *out = v[i];
    return true;
  }
  bool real(const char* s, const char* l, double* out) const {
    std::string t;
    if (!str(s, l, &t)) return false;
    *out = std::strtod(t.c_str(), nullptr);
    return true;
  }
  bool integer(const char* s, const char* l, int* out) const {
    std::string t;
    if (!str(s, l, &t)) return false;
    *out = static_cast<int>(std::strtol(t.c_str(), nullptr, 10));
    return true;
  }
};

// -------------------------------------------------------------------- CSV
// csvr::get_real (io/csvr.cpp:56-110): values are emitted only at ',';
// '#' comments to end of line; a character outside digits . , e - +
// discards up to and including the next ','; strtold then narrowing.
std::vector<double> read_reals(const std::string& path, bool* ok) {
  std::ifstream f(path);
  *ok = static_cast<bool>(f);
  std::vector<double> out;
  if (!f) return out;
  std::string tok;
  char c;
  while (f >> c) {
    if (c == '#') {
      f.ignore(1 << 30, '\n');
      tok.clear();
    } else if (!((c >= '0' && c <= '9') || c == '.' || c == ',' || c == '\n' || c == 'e' || c == '-' || c == '+')) {
      f.ignore(1 << 30, ',');
      tok.clear();
    } else if (c != ',' && c != '\n') {
      tok += c;
    } else if (!tok.empty()) {
      char* end = nullptr;
      long double v = std::strtold(tok.c_str(), &end);
      if (*end) {
        std::cout << "CSV parsing failed. Invalid data contained at line (unknown).\n";
        return out;
      }
      out.push_back(static_cast<double>(v));
      tok.clear();
    }
  }
  return out;
}

// -------------------------------------------------------------------- XML
// Enough XML for analyses.xml and graphml: elements, attributes, text,
// comments and declarations.
struct Node {
  std::string tag, text;
  std::map<std::string, std::string> attr;
  std::vector<Node> kids;
  const Node* child(const std::string& t) const {
    for (const Node& k : kids)
      if (k.tag == t) return &k;
    return nullptr;
  }
};

struct XmlReader {
  const std::string& s;
  size_t i = 0;
  explicit XmlReader(const std::string& text) : s(text) {}
  void skip_misc() {
    for (;;) {
      while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
      if (s.compare(i, 4, "<!--") == 0) {
        size_t e = s.find("-->", i);
        i = e == std::string::npos ? s.size() : e + 3;
      } else if (s.compare(i, 2, "<?") == 0 || s.compare(i, 2, "<!") == 0) {
        size_t e = s.find('>', i);
        i = e == std::string::npos ? s.size() : e + 1;
      } else {
        return;
      }
    }
  }
  bool element(Node& n) {
    skip_misc();
    if (i >= s.size() || s[i] != '<') return false;
    ++i;
    size_t b = i;
    while (i < s.size() && !std::isspace(static_cast<unsigned char>(s[i])) && s[i] != '>' && s[i] != '/') ++i;
    n.tag = s.substr(b, i - b);
    for (;;) {
      while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
      if (i >= s.size()) return false;
      if (s[i] == '/') {
        i = s.find('>', i) + 1;
        return true;
      }
      if (s[i] == '>') {
        ++i;
        break;
      }
      size_t k = i;
      while (i < s.size() && s[i] != '=' && !std::isspace(static_cast<unsigned char>(s[i]))) ++i;
      std::string key = s.substr(k, i - k);
      i = s.find_first_of("\"'", i);
      if (i == std::string::npos) return false;
      char q = s[i++];
      size_t e = s.find(q, i);
      n.attr[key] = s.substr(i, e - i);
      i = e + 1;
    }
    for (;;) {
      size_t lt = s.find('<', i);
      if (lt == std::string::npos) return false;
      n.text += s.substr(i, lt - i);
      i = lt;
      if (s.compare(i, 2, "</") == 0) {
        i = s.find('>', i) + 1;
        return true;
      }
      if (s.compare(i, 4, "<!--") == 0 || s.compare(i, 2, "<?") == 0) {
        skip_misc();
        continue;
      }
      Node k;
      if (!element(k)) return false;
      n.kids.push_back(std::move(k));
    }
  }
};

bool parse_xml_file(const std::string& path, Node* root) {
  std::ifstream f(path);
  if (!f) return false;
  std::stringstream ss;
  ss << f.rdbuf();
  std::string text = ss.str();
  XmlReader r(text);
  return r.element(*root);
}

std::string trim(const std::string& x) {
  size_t b = x.find_first_not_of(" \t\r\n"), e = x.find_last_not_of(" \t\r\n");
  return b == std::string::npos ? std::string() : x.substr(b, e - b + 1);
}

// ------------------------------------------------------------------ tissue
struct Graph {
  std::vector<std::set<int>> out;  // out-neighbours, ascending (std::set)
};

// create_default_graph (Sim_Initializer.hpp:103-136).
Graph default_graph(int n, int w) {
  Graph g;
  g.out.resize(n);
  for (int i = 0; i < n; ++i) {
    bool former = i % w == 0, latter = (i + 1) % w == 0, even = i % 2 == 0;
    int la = (former || !even) ? w - 1 : -1;
    int ra = !(latter || even) ? w + 1 : 1;
    int top = (i - w + n) % n, bottom = (i + w) % n, bottom_right = (i + ra) % n, top_left = (i + la) % n;
    int top_right = (i - w + ra + n) % n, bottom_left = (i - w + la + n) % n;
    std::vector<int> nb;
    if (former) nb = {top, top_left, top_right, bottom_left};
    else if (latter) nb = {top, top_right, bottom_right, bottom};
    else nb = {top_right, bottom_right, bottom, top_left, bottom_left};
    for (int x : nb) g.out[i].insert(std::abs(x));
  }
  return g;
}

// A graph whose vertex ids are not 0..n-1: DENSE indexes cells by id
// (sim/base.hpp:266-280), so ids are mapped to their rank here.
Graph from_edges(const std::set<long>& verts, const std::vector<std::pair<long, long>>& edges) {
  std::map<long, int> rank;
  for (long v : verts) rank.emplace(v, static_cast<int>(rank.size()));
  Graph g;
  g.out.resize(rank.size());
  for (auto& e : edges) g.out[rank[e.first]].insert(rank[e.second]);
  return g;
}

// NGraph's istream reader (ngraph/ngraph.hpp:942-1033): one vertex or one
// directed edge per line, '%'/'#' comments; a last line without a newline
// is dropped, as getline's eof check there does.
bool read_edge_list(const std::string& path, Graph* g) {
  std::ifstream f(path);
  if (!f) return false;
  std::set<long> verts;
  std::vector<std::pair<long, long>> edges;
  std::string line;
  for (;;) {
    bool got = false;
    while (std::getline(f, line)) {
      if (line.size() >= 1) {
        got = true;
        break;
      }
    }
    if (!got || f.eof()) break;
    if (line[0] == '%' || line[0] == '#') continue;
    std::istringstream L(line);
    long a = 0, b = 0;
    L >> a;
    verts.insert(a);
    if (!L.eof()) {
      if (!(L >> b)) b = 0;
      verts.insert(b);
      edges.emplace_back(a, b);
    }
  }
  *g = from_edges(verts, edges);
  return true;
}

// parse_graphml (Sim_Initializer.hpp:65-101): <edge> elements under <graph>
// (or <graph><edges>), vertex1/vertex2 or source/target, a leading 'n'
// stripped, self-loops dropped.
bool read_graphml(const std::string& path, Graph* g) {
  Node root;
  if (!parse_xml_file(path, &root)) return false;
  const Node* graph = root.child("graph");
  if (!graph) return false;
  const Node* holder = graph->child("edges") ? graph->child("edges") : graph;
  std::set<long> verts;
  std::vector<std::pair<long, long>> edges;
  for (const Node& e : holder->kids) {
    if (e.tag != "edge") continue;
    auto get = [&](const char* k) { auto it = e.attr.find(k); return it == e.attr.end() ? std::string() : it->second; };
    std::string b = get("vertex1"), t = get("vertex2");
    if (b.empty()) { b = get("source"); t = get("target"); }
    if (!b.empty() && b[0] == 'n') { b.erase(0, 1); t.erase(0, 1); }
    long x = 0, y = 0;
    try {
      x = std::stol(b);
      y = std::stol(t);
    } catch (const std::exception&) {
      return false;  // a vertex id that is not a number: the graph is invalid
    }
    if (x == y) continue;
    verts.insert(x);
    verts.insert(y);
    edges.emplace_back(x, y);
  }
  *g = from_edges(verts, edges);
  return true;
}

// ---------------------------------------------------------------- species
std::vector<int> species_list(const std::string& text, int ns) {
  std::vector<int> out;
  if (text == "*" || text.empty() || text == "all") {
    for (int i = 0; i < ns; ++i) out.push_back(i);
    return out;
  }
  std::istringstream st(text);
  std::string tok;
  while (std::getline(st, tok, ',')) {
    tok = trim(tok);
    int found = -1;
    for (int i = 0; i < ns; ++i)
      if (tok == dense_model_specie_name(i)) found = i;
    if (found < 0) {
      std::cout << "Warning: unknown species \"" << tok << "\" ignored\n";
      continue;
    }
    out.push_back(found);
  }
  return out;
}

// DENSE's NaNs come out of x86 arithmetic with the sign bit set and are
// printed "-nan"; the engine writes every NaN the same way.
struct Out {
  std::ostream* os;
  Out& operator<<(double x) {
    if (std::isnan(x)) *os << "-nan";
    else *os << x;
    return *this;
  }
  template <typename T>
  Out& operator<<(const T& x) {
    *os << x;
    return *this;
  }
};

std::string file_add_num(std::string name, unsigned no) {  // run_simulation.hpp:54-63
  std::string num = std::to_string(no);
  if (num.size() < 4) num.insert(0, 4 - num.size(), '0');
  size_t dot = std::min(name.find_last_of('.'), name.size());
  name.insert(dot, "_" + num);
  return name;
}

struct Entry {
  dense_analysis_desc d;
  std::vector<int> species;
  std::string out;
};

void usage() {
  std::cout << "[-h | --help | --usage]          Print this help.\n"
               "[-p | --param-sets]    <string> Parameter sets CSV.\n"
               "[-b | --perturbations] <string|Real> Perturbation factors entering the history sizing.\n"
               "[-e | --data-export]   <string> Trajectory export CSV.\n"
               "[-i | --data-import]   <string> Analyse a trajectory export instead of simulating (with -t, -u).\n"
               "[-o | --specie-option] <string> Species to export / analyse.\n"
               "[-a | --analysis]      <string> Analysis XML.\n"
               "[-c | --cell-total]       <int> Cells.\n"
               "[-w | --tissue-width]     <int> Tissue width.\n"
               "[-f | --cell-graph]    <string> Cell graph file (edge list or graphml).\n"
               "[-s | --step-size]       <Real> Euler step in minutes.\n"
               "[-t | --time-total]      <Real> Simulated minutes.\n"
               "[-u | --anlys-intvl]     <Real> Minutes between analysis samples.\n"
               "[-v | --time-col]               Time column in the export.\n"
               "[-d | --initial-conc]  <string> Initial concentrations CSV.\n"
               "[-N | --test-run]               No output.\n"
               "[--precision fp64|fp32] [--device <n>]\n";
}

}  // namespace

// The analyses of a run (parse_analysis_entries.hpp:64-126): analyses.xml
// entries (-a), else the trajectory export (-e), else a Basic analysis of
// every species and cell unless -N.  False when the XML cannot be read.
static bool parse_entries(const Args& A, int cells, int NS, std::vector<Entry>* entries, bool* time_col) {
  std::string default_sp;
  A.str("o", "specie-option", &default_sp);
  std::string xml_path, export_path;
  // DENSE reads -v as a flag with a value (parse_analysis_entries.hpp:365):
  // it is on only when another argument follows it
  std::string time_col_arg;
  *time_col = A.str("v", "time-col", &time_col_arg);
  if (A.str("a", "analysis", &xml_path)) {
    Node root;
    if (!parse_xml_file(xml_path, &root)) {
      std::cout << "Error: could not read analysis file " << xml_path << "\n";
      return false;
    }
    for (const Node& an : root.kids) {
      if (an.tag != "anlys") continue;
      auto text = [&](const char* k) { const Node* c = an.child(k); return c ? trim(c->text) : std::string(); };
      std::string type = an.attr.count("type") ? an.attr.at("type") : "";
      Entry e;
      std::memset(&e.d, 0, sizeof(e.d));
      e.species = species_list(text("species"), NS);
      e.d.cell_start = static_cast<int>(std::stold(text("cell-start")));
      e.d.cell_end = static_cast<int>(std::stold(text("cell-end")));
      e.d.time_start = static_cast<double>(std::stold(text("time-start")));
      e.d.time_end = static_cast<double>(std::stold(text("time-end")));
      e.out = text("out-file");
      if (type == "basic") {
        e.d.kind = DENSE_ANALYSIS_BASIC;
      } else if (type == "oscillation") {
        e.d.kind = DENSE_ANALYSIS_OSCILLATION;
        e.d.win_range = static_cast<double>(std::stold(text("win-range")));
        e.d.anlys_intvl = static_cast<double>(std::stold(text("anlys-intvl")));
      } else {
        std::cout << "Warning: Skipping unknown analysis type \"" << type << "\"\n";
        continue;
      }
      if (e.d.cell_start < 0 || e.d.cell_end > cells || e.d.cell_end < e.d.cell_start) {
        std::cout << "Warning: skipping analysis of cells " << e.d.cell_start << "-" << e.d.cell_end
                  << ", outside the " << cells << "-cell tissue\n";
        continue;
      }
      entries->push_back(e);
    }
  } else if (A.str("e", "data-export", &export_path) && !export_path.empty()) {
    Entry e;
    std::memset(&e.d, 0, sizeof(e.d));
    e.d.kind = DENSE_ANALYSIS_TRAJECTORY;
    e.species = species_list(default_sp, NS);
    e.d.cell_start = 0;
    e.d.cell_end = cells;
    e.d.time_start = 0;
    e.d.time_end = INFINITY;
    e.out = export_path;
    entries->push_back(e);
  } else if (!A.has("N", "test-run")) {
    std::cout << "Warning: performing basic analysis only.  Did you mean to use the [-e | --data-export] and/or "
                 "[-a | --analysis] flag(s)? (use -N to suppress this error)\n";
    Entry e;
    std::memset(&e.d, 0, sizeof(e.d));
    e.d.kind = DENSE_ANALYSIS_BASIC;
    e.species = species_list(default_sp, NS);
    e.d.cell_start = 0;
    e.d.cell_end = cells;
    e.d.time_start = 0;
    e.d.time_end = INFINITY;
    entries->push_back(e);
  }
  return true;
}

// Every analysis' output of every set that was not dropped, as DENSE's
// run_simulation shows them (run_simulation.hpp:113-121, 159-163).
static void write_outputs(dense_engine* eng, const std::vector<Entry>& entries, int num_sets, int NS, bool time_col,
                          const std::vector<int32_t>& status) {
  for (int s = 0; s < num_sets; ++s) {
    if (status[s] & DENSE_SET_DROPPED) continue;  // run_simulation drops bad sets (run_simulation.hpp:131-150)
    for (size_t ai = 0; ai < entries.size(); ++ai) {
      const Entry& e = entries[ai];
      std::ofstream file;
      std::ostream* os = &std::cout;
      if (!e.out.empty()) {
        file.open(num_sets == 1 ? e.out : file_add_num(e.out, static_cast<unsigned>(s)));
        os = &file;
      }
      Out out{os};
      const int n = e.d.num_species, m = e.d.cell_end - e.d.cell_start;
      if (e.d.kind == DENSE_ANALYSIS_TRAJECTORY) {
        int samples = 0;
        dense_engine_read_trajectory(eng, static_cast<int>(ai), s, nullptr, nullptr, 0, &samples);
        std::vector<double> times(samples), vals(static_cast<size_t>(samples) * n * m);
        dense_engine_read_trajectory(eng, static_cast<int>(ai), s, times.data(), vals.data(), samples, &samples);
        for (int k = 0; k < samples; ++k) {
          if (k == 0) {  // csvw_sim::update header (io/csvw_sim.ipp:19-60)
            out << "\n# This file can be used as a template for user-created/modified analysis inputs in the "
                   "context of this particular model for these particular command-line arguments.\n"
                << "# The row after next MUST remain in the file in order for it to be parsable by the CSV "
                   "reader. They indicate the following:\ncell-total, time-start, time-col, cell-start, "
                   "cell-end, specie-option,\n"
                << e.d.cell_end << ',' << times[0] << ',' << time_col << ',' << e.d.cell_start << ','
                << e.d.cell_end << ',';
            for (int sp = 0; sp < NS; ++sp) {
              bool on = false;
              for (int x : e.species) on = on || x == sp;
              out << (on ? 1.0 : 0.0) << ',';
            }
            out << "\n\n";
            if (time_col) out << "Time,";
            for (int x : e.species) out << dense_model_specie_name(x) << ',';
            out << '\n';
          }
          for (int c = 0; c < m; ++c) {
            if (time_col) {
              if (c == 0) out << "Time: " << times[k] << ',';
              else out << ',';
            }
            for (int i = 0; i < n; ++i) out << vals[(static_cast<size_t>(k) * n + i) * m + c] << ',';
            out << '\n';
          }
          if (m > 0) out << '\n';
        }
        // run_simulation's final show() of csvw_sim is Analysis<>::show
        // (measurement/base.hpp:40-51)
        out << "# Showing cells " << e.d.cell_start << '-' << e.d.cell_end << " until "
            << (samples > 0 ? times[samples - 1] : 0.0) << " min\n";
        continue;
      }
      double time = 0;
      int samples = 0;
      if (e.d.kind == DENSE_ANALYSIS_BASIC) {
        std::vector<double> mins(n), sums(n), maxs(n);
        dense_engine_read_basic(eng, static_cast<int>(ai), s, mins.data(), sums.data(), maxs.data(), nullptr,
                                nullptr, nullptr, &samples, &time);
        // Analysis<>::show + BasicAnalysis::show (base.hpp:40-51, basic.ipp:61-75)
        out << "# Showing cells " << e.d.cell_start << '-' << e.d.cell_end;
        if (e.d.time_start != 0.0) out << " between " << e.d.time_start << " min and ";
        else out << " until ";
        out << time << " min\n";
        out << "Species,Minimum Concentration,Mean Concentration,Maximum Concentration\n";
        for (int sp : e.species) {
          // DENSE indexes these vectors by species id (basic.ipp:69-72)
          double mn = NAN, mean = NAN, mx = NAN;
          if (sp < n) {
            mn = mins[sp];
            mx = maxs[sp];
            mean = sums[sp] / (samples * (e.d.cell_end - e.d.cell_start));
          }
          out << dense_model_specie_name(sp) << ',' << mn << ',' << mean << ',' << mx << '\n';
        }
      } else {
        std::vector<double> amps(static_cast<size_t>(n) * m), pers(amps.size()), peaks(amps.size());
        std::vector<int> ncrit(amps.size());
        dense_engine_read_oscillation(eng, static_cast<int>(ai), s, amps.data(), pers.data(), peaks.data(),
                                      ncrit.data(), &samples, &time);
        out << "# Showing cells " << e.d.cell_start << '-' << e.d.cell_end;
        if (e.d.time_start != 0.0) out << " between " << e.d.time_start << " min and ";
        else out << " until ";
        out << time << " min\n";
        for (int c = 0; c < m; ++c) {  // OscillationAnalysis::show (oscillation.ipp:30-77)
          out << "\n# Showing cell " << (c + e.d.cell_start) << "\nSpecies";
          for (int sp : e.species) out << ',' << dense_model_specie_name(sp);
          out << "\navg peak,";
          for (int i = 0; i < n; ++i) out << peaks[static_cast<size_t>(i) * m + c] << ',';
          out << "\navg amp,";
          for (int i = 0; i < n; ++i) out << amps[static_cast<size_t>(i) * m + c] << ',';
          out << "\navg per,";
          for (int i = 0; i < n; ++i) out << pers[static_cast<size_t>(i) * m + c] << ',';
        }
      }
    }
  }
}

// A trajectory export (csvw_sim, io/csvw_sim.ipp:17-91: what -e writes)
// read back for -i: the header row (cell-total, time-start, time-col,
// cell-start, cell-end, one 0/1 flag per species), the row of column names
// (the value columns' species in file order -- csvw_sim writes them in the
// -o order -- after an optional Time and Cell column), then cell-end -
// cell-start rows of values per sample.  Numbers are read as DENSE reads
// them (strtold, then double).  samples is [k][NS][cell-total], NaN where
// the file holds no value.
struct Import {
  int cells = 0, cell_start = 0, cell_end = 0, time_col = 0, k = 0;
  double time_start = 0;
  std::vector<int> species;  // value columns, file order
  std::vector<double> samples;
};

static bool read_import(const std::string& path, int NS, Import* im, std::string* err) {
  std::ifstream f(path);
  if (!f) {
    *err = "CSV file input failed. CSV file '" + path + "' not found or open.";
    return false;
  }
  auto split = [](const std::string& ln) {
    std::vector<std::string> out;
    std::string cur;
    for (char c : ln) {
      if (c == ',') {
        out.push_back(trim(cur));
        cur.clear();
      } else {
        cur += c;
      }
    }
    if (!trim(cur).empty()) out.push_back(trim(cur));
    return out;
  };
  auto number = [](const std::string& t, double* v) {
    char* end = nullptr;
    const long double x = std::strtold(t.c_str(), &end);
    *v = static_cast<double>(x);
    return !t.empty() && end && *end == 0;
  };
  std::vector<std::string> body;
  std::string ln;
  while (std::getline(f, ln)) {
    const std::string t = trim(ln);
    if (!t.empty() && t[0] != '#') body.push_back(t);
  }
  if (body.size() < 3 || body[0].compare(0, 10, "cell-total") != 0) {
    *err = "not a trajectory export (no cell-total header row): " + path;
    return false;
  }
  const std::vector<std::string> head = split(body[1]);
  if (static_cast<int>(head.size()) != 5 + NS) {
    *err = "trajectory header has " + std::to_string(head.size()) + " fields, expected " + std::to_string(5 + NS);
    return false;
  }
  std::vector<double> h(head.size());
  for (size_t i = 0; i < head.size(); ++i)
    if (!number(head[i], &h[i])) {
      *err = "trajectory header field '" + head[i] + "' is not a number";
      return false;
    }
  im->cells = static_cast<int>(h[0]);
  im->time_start = h[1];
  im->time_col = static_cast<int>(h[2]);
  im->cell_start = static_cast<int>(h[3]);
  im->cell_end = static_cast<int>(h[4]);
  if (im->cells <= 0 || im->cell_start < 0 || im->cell_end > im->cells || im->cell_end <= im->cell_start) {
    *err = "trajectory header's cell range is invalid";
    return false;
  }
  std::vector<std::string> names = split(body[2]);
  size_t skip = 0;
  while (skip < names.size() && (names[skip] == "Time" || names[skip] == "Cell")) ++skip;
  std::vector<bool> flagged(NS), seen(NS);
  for (int i = 0; i < NS; ++i) flagged[i] = h[5 + i] != 0.0;
  for (size_t j = skip; j < names.size(); ++j) {
    int id = -1;
    for (int i = 0; i < NS; ++i)
      if (names[j] == dense_model_specie_name(i)) id = i;
    if (id < 0 || !flagged[id] || seen[id]) {
      *err = "trajectory column '" + names[j] + "' is not one of the header's species";
      return false;
    }
    seen[id] = true;
    im->species.push_back(id);
  }
  if (seen != flagged) {
    *err = "trajectory columns do not match the header's species flags";
    return false;
  }
  const int m = im->cell_end - im->cell_start, ncol = static_cast<int>(im->species.size());
  std::vector<double> rows;
  for (size_t r = 3; r < body.size(); ++r) {
    std::vector<std::string> v = split(body[r]);
    // the Time (and Cell) cells come first; only a sample's first row
    // carries its time, the others leave the cell empty
    if (v.size() == static_cast<size_t>(ncol) + skip) v.erase(v.begin(), v.begin() + skip);
    else if (skip > 0 && v.size() + 1 == static_cast<size_t>(ncol) + skip && body[r][0] == ',')
      v.erase(v.begin(), v.begin() + (skip - 1));
    if (static_cast<int>(v.size()) != ncol) {
      *err = "trajectory row " + std::to_string(r) + " holds " + std::to_string(v.size()) + " values, expected " +
             std::to_string(ncol);
      return false;
    }
    for (const std::string& t : v) {
      double x;
      if (!number(t, &x)) {
        *err = "trajectory value '" + t + "' is not a number";
        return false;
      }
      rows.push_back(x);
    }
  }
  const size_t per = static_cast<size_t>(m) * ncol;
  if (per == 0 || rows.size() % per) {
    *err = "trajectory rows are not whole samples of " + std::to_string(m) + " cells";
    return false;
  }
  im->k = static_cast<int>(rows.size() / per);
  im->samples.assign(static_cast<size_t>(im->k) * NS * im->cells, NAN);
  for (int k = 0; k < im->k; ++k)
    for (int c = 0; c < m; ++c)
      for (int j = 0; j < ncol; ++j)
        im->samples[(static_cast<size_t>(k) * NS + im->species[j]) * im->cells + im->cell_start + c] =
            rows[(static_cast<size_t>(k) * m + c) * ncol + j];
  return true;
}

static int run_cli(int argc, char** argv) {
  Args A;
  A.v.assign(argv + 1, argv + argc);
  if (A.has("h", "help") || A.has("H", "usage") || argc == 1) {
    usage();
    return EXIT_SUCCESS;
  }
  // DENSE flags outside this command: the stochastic seed (-r) and the
  // colour switch (-n) change nothing here and are accepted; gradients (-g)
  // are undefined in DENSE (simulation_width_ is 0 when gradient_index is
  // taken modulo it, sim/base.cpp:22-31), so they are refused rather than
  // ignored
  if (A.has("g", "gradients")) {
    std::cout << "Error: [-g | --gradients] is not supported (DENSE's gradient path divides by the tissue width "
                 "before it is set); give per-cell parameters instead.\n";
    return EXIT_FAILURE;
  }
  dense_model_info mi;
  dense_model_get_info(&mi);
  const int NS = mi.num_species, NP = mi.num_params, NR = mi.num_reactions;

  // -i: analysis of an imported trajectory (main.cpp:160-175): no
  // simulation; the analyses see the file's samples, one per chunk of -u
  // minutes from the file's start time, for -t minutes (or as many samples
  // as the file holds).  DENSE's own reader for it (CSV_Streamed_Simulation,
  // io/csvr_sim.cpp:87-96) calls itself and never returns.
  std::string import_path;
  if (A.str("i", "data-import", &import_path)) {
    double time_total = 0, anlys_intvl = 0;
    if (!(A.real("t", "time-total", &time_total) && A.real("u", "anlys-intvl", &anlys_intvl)) ||
        !(anlys_intvl > 0.0)) {
      std::cout << "No time-total or anlys-intvl for CSV Simulation (fix in future)\n";
      return EXIT_FAILURE;
    }
    Import im;
    std::string err;
    if (!read_import(import_path, NS, &im, &err)) {
      std::cout << "Error: " << err << "\n";
      return EXIT_FAILURE;
    }
    std::vector<Entry> entries;
    bool time_col = false;
    if (!parse_entries(A, im.cells, NS, &entries, &time_col)) return EXIT_FAILURE;
    for (Entry& e : entries) {
      for (int sp : e.species) {
        bool held = false;
        for (int x : im.species) held = held || x == sp;
        if (!held) {
          std::cout << "Error: the imported trajectory holds no " << dense_model_specie_name(sp) << "\n";
          return EXIT_FAILURE;
        }
      }
      if (e.d.cell_start < im.cell_start || e.d.cell_end > im.cell_end) {
        std::cout << "Error: analysis of cells " << e.d.cell_start << "-" << e.d.cell_end
                  << " outside the imported cells " << im.cell_start << "-" << im.cell_end << "\n";
        return EXIT_FAILURE;
      }
      e.d.num_species = static_cast<int>(e.species.size());
      e.d.species = e.species.data();
    }
    std::vector<dense_analysis_desc> descs;
    for (Entry& e : entries) descs.push_back(e.d);
    int device = 0;
    A.integer("device", "device", &device);
    // one set of the file's cells, no neighbours; its parameters are never used
    std::vector<int> off(im.cells + 1, 0), ids(1, 0);
    std::vector<double> prm(NP, 0.0);
    dense_set_desc set{};
    set.num_cells = im.cells;
    set.nbr_offsets = off.data();
    set.nbr_ids = ids.data();
    set.set_params = prm.data();
    set.duration = time_total;
    dense_run_desc run{DENSE_FP64, anlys_intvl, anlys_intvl, static_cast<int>(descs.size()), descs.data(), device};
    dense_engine* eng = nullptr;
    const double chunks = std::ceil(time_total / anlys_intvl);  // run_simulation.hpp:127-130
    const int k = static_cast<int>(std::min<double>(chunks, im.k));
    if (dense_engine_create(&run, 1, &set, &eng) != DENSE_OK ||
        dense_engine_analyze_samples(eng, 0, im.samples.data(), k, im.time_start) != DENSE_OK) {
      std::cout << "Error: " << dense_last_error() << "\n";
      return EXIT_FAILURE;
    }
    std::vector<int32_t> status(1);
    dense_engine_status(eng, status.data());
    write_outputs(eng, entries, 1, NS, time_col, status);
    dense_engine_destroy(eng);
    return EXIT_SUCCESS;
  }

  double time_total = 0, anlys_intvl = 0, step_size = 0;
  std::string param_path;
  bool ok = A.real("t", "time-total", &time_total);
  ok = A.real("u", "anlys-intvl", &anlys_intvl) && ok;
  ok = A.str("p", "param-sets", &param_path) && ok;
  if (!ok) {
    std::cout << "Error: Your current set of command line arguments produces a useless state. (No inputs are "
                 "specified.)\n";
    return EXIT_FAILURE;
  }
  if (!A.real("s", "step-size", &step_size) || step_size == 0.0) {
    std::cout << "Error: the deterministic engine needs [-s | --step-size].\n";
    return EXIT_FAILURE;
  }
  bool csv_ok;
  std::vector<double> pvals = read_reals(param_path, &csv_ok);
  if (!csv_ok) {
    std::cout << "CSV file input failed. CSV file '" << param_path << "' not found or open.\n";
    return EXIT_FAILURE;
  }
  if (pvals.size() % NP) {
    std::cout << "ERROR: Partial set encountered at end of Parameter Sets CSV file.\n";
    return EXIT_FAILURE;
  }
  const int num_sets = static_cast<int>(pvals.size() / NP);

  // tissue (arg_parse.hpp:127-169)
  int cells = 0, width = 0;
  std::string graph_path;
  bool c_flag = A.integer("c", "cell-total", &cells), w_flag = A.integer("w", "tissue-width", &width);
  bool f_flag = A.str("f", "cell-graph", &graph_path);
  Graph g;
  if (w_flag && c_flag && !f_flag) {
    if (cells <= 0 || width <= 0 || width > cells) {
      std::cout << "Error: invalid cell total or tissue width.\n";
      return EXIT_FAILURE;
    }
    g = default_graph(cells, width);
  } else if (f_flag && !c_flag && !w_flag) {
    bool gok = graph_path.find("graphml") != std::string::npos ? read_graphml(graph_path, &g)
                                                              : read_edge_list(graph_path, &g);
    if (!gok || g.out.empty()) {
      std::cout << "Error: Cell graph from " << graph_path << " is invalid.\n";
      return EXIT_FAILURE;
    }
    cells = static_cast<int>(g.out.size());
  } else {
    std::cout << "Error: Either specify a cell total with [-c | --cell-total] and a width with [-w | "
                 "--tissue-width] or provide a cell graph file with [-f | --cell-graph].\n";
    return EXIT_FAILURE;
  }
  std::vector<int> off{0}, ids;
  for (auto& nb : g.out) {
    for (int x : nb) ids.push_back(x);
    off.push_back(static_cast<int>(ids.size()));
  }

  // initial concentrations (conc_vector, Sim_Initializer.hpp:138-157)
  std::vector<double> conc;
  std::string conc_path;
  // (DENSE dereferences a failed reader here and crashes; the file must open)
  if (A.str("d", "initial-conc", &conc_path)) {
    conc = read_reals(conc_path, &csv_ok);
    if (!csv_ok) {
      std::cout << "CSV file input failed. CSV file '" << conc_path << "' not found or open.\n";
      return EXIT_FAILURE;
    }
    conc.resize(NS, 0.0);
  }
  // -b: one global factor or a per-reaction CSV (history sizing only)
  std::vector<double> pert;
  std::string pb;
  if (A.str("b", "perturbations", &pb)) {
    char* end = nullptr;
    double v = std::strtod(pb.c_str(), &end);
    if (end && *end == 0) pert.assign(NR, v);
    else {
      pert = read_reals(pb, &csv_ok);
      if (!csv_ok) {
        std::cout << "CSV file input failed. CSV file '" << pb << "' not found or open.\n";
        return EXIT_FAILURE;
      }
      pert.resize(NR, 0.0);
    }
  }

  std::vector<Entry> entries;
  bool time_col = false;
  if (!parse_entries(A, cells, NS, &entries, &time_col)) return EXIT_FAILURE;
  for (Entry& e : entries) {
    e.d.num_species = static_cast<int>(e.species.size());
    e.d.species = e.species.data();
  }
  std::vector<dense_analysis_desc> descs;
  for (Entry& e : entries) descs.push_back(e.d);

  std::string prec = "fp64";
  A.str("precision", "precision", &prec);
  int device = 0;
  A.integer("device", "device", &device);
  std::vector<dense_set_desc> sets(num_sets);
  for (int s = 0; s < num_sets; ++s) {
    sets[s].num_cells = cells;
    sets[s].nbr_offsets = off.data();
    sets[s].nbr_ids = ids.data();
    sets[s].set_params = pvals.data() + static_cast<size_t>(s) * NP;
    sets[s].cell_params = nullptr;
    sets[s].init_conc = conc.empty() ? nullptr : conc.data();
    sets[s].perturb = pert.empty() ? nullptr : pert.data();
    sets[s].duration = time_total;
  }
  dense_run_desc run{prec == "fp32" ? DENSE_FP32_KAHAN : DENSE_FP64, step_size, anlys_intvl,
                     static_cast<int>(descs.size()), descs.data(), device};
  dense_engine* eng = nullptr;
  if (dense_engine_create(&run, num_sets, sets.data(), &eng) != DENSE_OK) {
    std::cout << "Error: " << dense_last_error() << "\n";
    return EXIT_FAILURE;
  }
  if (dense_engine_run(eng, -1, nullptr) != DENSE_OK || dense_engine_sync(eng) != DENSE_OK) {
    std::cout << "Error: " << dense_last_error() << "\n";
    return EXIT_FAILURE;
  }
  std::vector<int32_t> status(num_sets);
  dense_engine_status(eng, status.data());

  write_outputs(eng, entries, num_sets, NS, time_col, status);
  dense_engine_destroy(eng);
  return EXIT_SUCCESS;
}

int main(int argc, char** argv) {
  // a malformed number in an input file (std::stold / std::stol on an
  // analysis XML value or a graph vertex id) ends the run with a message;
  // DENSE lets the exception terminate the process
  try {
    return run_cli(argc, argv);
  } catch (const std::exception& e) {
    std::cout << "Error: malformed input (" << e.what() << ").\n";
    return EXIT_FAILURE;
  }
}
