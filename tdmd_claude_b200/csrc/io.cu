// io.cu -- the file formats around the path, native: LAMMPS `atomic` data
// files, `dump custom id type x y z fx fy fz` force dumps and the DYNAMO
// setfl EAM layout (host code only; no device work).
//
// Reference interfaces (tdmd_Claude):
//  * read_lammps_data (src/io/lammps_data_reader.cpp:33-204): the first line
//    is a title; header lines up to the first section keyword give
//    "N atoms", "N atom types" and "lo hi xlo xhi" (y, z); a section keyword
//    is followed by one skipped line, then its records, blank lines inside a
//    section are skipped; "Atoms" records are "id type x y z" stored at
//    index id-1, "Velocities" "id vx vy vz", "Masses" "type mass" into
//    masses[ntypes + 1] (default 1); a later line whose first character is
//    upper case starts the next section; other sections are skipped.
//  * read_lammps_dump (src/io/dump_reader.cpp:15-55): the count after
//    "ITEM: NUMBER OF ATOMS", records after "ITEM: ATOMS", sorted by id.
//  * write_lammps_force_dump (src/drivers/tdmd_main.cpp:65-95): TIMESTEP,
//    NUMBER OF ATOMS, BOX BOUNDS pp pp pp, ATOMS id type x y z fx fy fz,
//    17 significant digits.
//  * setfl (src/potentials/eam_alloy.cpp:90-192): 3 comment lines, the
//    element line, the grid line, per element a header line then Nrho F and
//    Nr rho values, then Nr r*phi values per pair i <= j.
//
// One deliberate difference: where the reference would index out of its
// arrays (an atom id outside 1..N, a type outside 1..ntypes in Masses), these
// readers return TDMD_ERR_PARSE instead.
#include <algorithm>
#include <cctype>
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"
#include "eam_tables.cuh"
#include "tdmd_b200.h"

struct tdmd_system {
  int64_t natoms = 0;
  int32_t ntypes = 0;
  tdmd_box box{};
  std::vector<double> pos, vel;  // [3n]
  std::vector<int32_t> types, ids;
  std::vector<double> masses;  // [ntypes + 1], index 0 unused
};

namespace tdmd_b200 {
namespace {

std::string trim(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  const size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

bool begins(const std::string& s, const char* p) { return s.compare(0, std::strlen(p), p) == 0; }

[[noreturn]] void parse_fail(const std::string& msg) { throw Error{TDMD_ERR_PARSE, msg}; }

void read_data(const std::string& path, tdmd_system& st) {
  std::ifstream in(path);
  if (!in.is_open()) throw Error{TDMD_ERR_IO, "cannot open LAMMPS data file: " + path};
  std::string line;
  std::getline(in, line);  // title
  int64_t natoms = 0;
  int32_t ntypes = 0;
  bool box[3] = {false, false, false};
  bool at_section = false;
  while (std::getline(in, line)) {
    const std::string t = trim(line);
    if (t.empty()) continue;
    if (t == "Atoms" || t == "Velocities" || t == "Masses" || begins(t, "Atoms ") ||
        begins(t, "Pair Coeffs") || begins(t, "Bond Coeffs")) {
      at_section = true;
      break;
    }
    std::istringstream is(t);
    if (t.find("atoms") != std::string::npos) {
      is >> natoms;
      if (is.fail() || natoms <= 0) parse_fail("invalid atom count in header");
      continue;
    }
    if (t.find("atom types") != std::string::npos) {
      is >> ntypes;
      if (is.fail() || ntypes <= 0) parse_fail("invalid atom type count in header");
      continue;
    }
    static const char* kAxes[3] = {"xlo xhi", "ylo yhi", "zlo zhi"};
    for (int a = 0; a < 3; ++a)
      if (t.find(kAxes[a]) != std::string::npos) {
        is >> st.box.lo[a] >> st.box.hi[a];
        box[a] = true;
      }
  }
  if (natoms == 0) parse_fail("no atoms in data file");
  if (!box[0] || !box[1] || !box[2]) parse_fail("incomplete box definition");
  const size_t n = static_cast<size_t>(natoms);
  st.natoms = natoms;
  st.ntypes = ntypes;
  for (int a = 0; a < 3; ++a) st.box.periodic[a] = 1;
  st.pos.assign(3 * n, 0.0);
  st.vel.assign(3 * n, 0.0);
  st.types.assign(n, 0);
  st.ids.assign(n, 0);
  st.masses.assign(static_cast<size_t>(ntypes) + 1, 1.0);
  bool atoms_read = false;
  // Reads `count` non-blank records of the current section after skipping
  // the line that follows its keyword.
  auto records = [&](int64_t count, const char* what, auto&& take) {
    std::getline(in, line);
    for (int64_t k = 0; k < count; ++k) {
      if (!std::getline(in, line)) parse_fail(std::string("premature end in ") + what);
      const std::string t = trim(line);
      if (t.empty()) {
        --k;
        continue;
      }
      std::istringstream is(t);
      if (!take(is)) parse_fail(std::string("bad ") + what + " line: " + t);
    }
  };
  auto id_index = [&](int32_t id) -> size_t {
    if (id < 1 || id > natoms) parse_fail("atom id out of range 1..N: " + std::to_string(id));
    return static_cast<size_t>(id - 1);
  };
  auto section = [&]() {
    std::string s = trim(line);
    const size_t hash = s.find('#');
    if (hash != std::string::npos) s = trim(s.substr(0, hash));
    if (s == "Masses") {
      records(ntypes, "Masses", [&](std::istringstream& is) {
        int32_t t;
        double m;
        is >> t >> m;
        if (is.fail()) return false;
        if (t < 1 || t > ntypes) parse_fail("type out of range in Masses: " + std::to_string(t));
        st.masses[static_cast<size_t>(t)] = m;
        return true;
      });
    } else if (s == "Atoms") {
      records(natoms, "Atoms", [&](std::istringstream& is) {
        int32_t id, ty;
        double x, y, z;
        is >> id >> ty >> x >> y >> z;
        if (is.fail()) return false;
        const size_t i = id_index(id);
        st.ids[i] = id;
        st.types[i] = ty;
        st.pos[3 * i] = x;
        st.pos[3 * i + 1] = y;
        st.pos[3 * i + 2] = z;
        return true;
      });
      atoms_read = true;
    } else if (s == "Velocities") {
      records(natoms, "Velocities", [&](std::istringstream& is) {
        int32_t id;
        double vx, vy, vz;
        is >> id >> vx >> vy >> vz;
        if (is.fail()) return false;
        const size_t i = id_index(id);
        st.vel[3 * i] = vx;
        st.vel[3 * i + 1] = vy;
        st.vel[3 * i + 2] = vz;
        return true;
      });
    }
  };
  if (at_section) section();
  while (std::getline(in, line)) {
    const std::string t = trim(line);
    if (!t.empty() && std::isupper(static_cast<unsigned char>(t[0]))) section();
  }
  if (!atoms_read) parse_fail("no Atoms section found");
}

// Doubles with 17 significant digits (round-trip exact).
void put17(std::FILE* f, double v) { std::fprintf(f, "%.17g", v); }

struct File {
  std::FILE* f;
  explicit File(const char* path) : f(std::fopen(path, "w")) {
    if (!f) throw Error{TDMD_ERR_IO, std::string("cannot open for writing: ") + path};
  }
  ~File() {
    if (f) std::fclose(f);
  }
  void close() {
    const bool bad = std::ferror(f) != 0;
    const int rc = std::fclose(f);
    f = nullptr;
    if (bad || rc != 0) throw Error{TDMD_ERR_IO, "write error"};
  }
};

}  // namespace
}  // namespace tdmd_b200

using namespace tdmd_b200;

extern "C" {

int32_t tdmd_read_lammps_data(const char* path, tdmd_system** out) {
  return guarded([&] {
    TDMD_REQUIRE(path && out, "null argument");
    auto* s = new tdmd_system();
    try {
      read_data(path, *s);
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
  });
}

int32_t tdmd_system_destroy(tdmd_system* s) {
  delete s;
  return TDMD_OK;
}

int32_t tdmd_system_get(const tdmd_system* s, int64_t* natoms, int32_t* ntypes, tdmd_box* box,
                        const double** positions, const double** velocities,
                        const int32_t** types, const int32_t** ids, const double** masses) {
  return guarded([&] {
    TDMD_REQUIRE(s, "null handle");
    if (natoms) *natoms = s->natoms;
    if (ntypes) *ntypes = s->ntypes;
    if (box) *box = s->box;
    if (positions) *positions = s->pos.data();
    if (velocities) *velocities = s->vel.data();
    if (types) *types = s->types.data();
    if (ids) *ids = s->ids.data();
    if (masses) *masses = s->masses.data();
  });
}

int32_t tdmd_write_lammps_data(const char* path, const char* title, int64_t natoms,
                               int32_t ntypes, const tdmd_box* box, const double* positions,
                               const double* velocities, const int32_t* types,
                               const int32_t* ids, const double* masses) {
  return guarded([&] {
    TDMD_REQUIRE(path && box && positions && types, "null argument");
    TDMD_REQUIRE(natoms > 0 && ntypes > 0, "natoms and ntypes must be positive");
    File out(path);
    std::FILE* f = out.f;
    std::fprintf(f, "%s\n\n%" PRId64 " atoms\n%d atom types\n\n",
                 title ? title : "tdmd_claude_b200 data", natoms, ntypes);
    static const char* kAx[3] = {"x", "y", "z"};
    for (int a = 0; a < 3; ++a) {
      put17(f, box->lo[a]);
      std::fputc(' ', f);
      put17(f, box->hi[a]);
      std::fprintf(f, " %slo %shi\n", kAx[a], kAx[a]);
    }
    std::fprintf(f, "\nMasses\n\n");
    for (int t = 1; t <= ntypes; ++t) {
      std::fprintf(f, "%d ", t);
      put17(f, masses ? masses[t] : 1.0);
      std::fputc('\n', f);
    }
    std::fprintf(f, "\nAtoms # atomic\n\n");
    for (int64_t i = 0; i < natoms; ++i) {
      std::fprintf(f, "%d %d", ids ? ids[i] : static_cast<int32_t>(i + 1), types[i]);
      for (int a = 0; a < 3; ++a) {
        std::fputc(' ', f);
        put17(f, positions[3 * i + a]);
      }
      std::fputc('\n', f);
    }
    if (velocities) {
      std::fprintf(f, "\nVelocities\n\n");
      for (int64_t i = 0; i < natoms; ++i) {
        std::fprintf(f, "%d", ids ? ids[i] : static_cast<int32_t>(i + 1));
        for (int a = 0; a < 3; ++a) {
          std::fputc(' ', f);
          put17(f, velocities[3 * i + a]);
        }
        std::fputc('\n', f);
      }
    }
    out.close();
  });
}

int32_t tdmd_read_force_dump(const char* path, int64_t* natoms, int64_t capacity, int32_t* ids,
                             int32_t* types, double* positions, double* forces) {
  return guarded([&] {
    TDMD_REQUIRE(path && natoms, "null argument");
    std::ifstream in(path);
    if (!in.is_open()) throw Error{TDMD_ERR_IO, std::string("cannot open dump file: ") + path};
    std::string line;
    int64_t n = 0;
    bool atoms = false;
    while (std::getline(in, line)) {
      if (line.find("ITEM: NUMBER OF ATOMS") != std::string::npos) {
        if (!std::getline(in, line)) parse_fail("premature end of dump");
        char* end = nullptr;
        n = std::strtoll(line.c_str(), &end, 10);
        if (end == line.c_str()) parse_fail("bad atom count in dump: " + line);
      }
      if (line.find("ITEM: ATOMS") != std::string::npos) {
        atoms = true;
        break;
      }
    }
    if (n <= 0 || !atoms) parse_fail("no atoms in dump file");
    *natoms = n;
    if (!ids && !types && !positions && !forces) return;
    TDMD_REQUIRE(capacity >= n, "capacity smaller than the dump's atom count");
    struct Rec {
      int32_t id, type;
      double v[6];
    };
    std::vector<Rec> recs(static_cast<size_t>(n));
    for (int64_t k = 0; k < n; ++k) {
      if (!std::getline(in, line)) parse_fail("premature end of dump");
      std::istringstream is(line);
      Rec& r = recs[static_cast<size_t>(k)];
      is >> r.id >> r.type >> r.v[0] >> r.v[1] >> r.v[2] >> r.v[3] >> r.v[4] >> r.v[5];
      if (is.fail()) parse_fail("bad dump line: " + line);
    }
    std::stable_sort(recs.begin(), recs.end(),
                     [](const Rec& a, const Rec& b) { return a.id < b.id; });
    for (int64_t k = 0; k < n; ++k) {
      const Rec& r = recs[static_cast<size_t>(k)];
      if (ids) ids[k] = r.id;
      if (types) types[k] = r.type;
      for (int a = 0; a < 3; ++a) {
        if (positions) positions[3 * k + a] = r.v[a];
        if (forces) forces[3 * k + a] = r.v[3 + a];
      }
    }
  });
}

int32_t tdmd_write_force_dump(const char* path, int64_t step, int64_t natoms,
                              const tdmd_box* box, const int32_t* ids, const int32_t* types,
                              const double* positions, const void* forces,
                              int32_t force_precision) {
  return guarded([&] {
    TDMD_REQUIRE(path && box && types && positions && forces, "null argument");
    TDMD_REQUIRE(natoms >= 0, "natoms must be non-negative");
    TDMD_REQUIRE(force_precision == TDMD_FP64 || force_precision == TDMD_MIXED,
                 "unknown force precision");
    File out(path);
    std::FILE* f = out.f;
    std::fprintf(f, "ITEM: TIMESTEP\n%" PRId64 "\nITEM: NUMBER OF ATOMS\n%" PRId64 "\n", step,
                 natoms);
    std::fprintf(f, "ITEM: BOX BOUNDS pp pp pp\n");
    for (int a = 0; a < 3; ++a) {
      put17(f, box->lo[a]);
      std::fputc(' ', f);
      put17(f, box->hi[a]);
      std::fputc('\n', f);
    }
    std::fprintf(f, "ITEM: ATOMS id type x y z fx fy fz\n");
    const double* f64 = static_cast<const double*>(forces);
    const float* f32 = static_cast<const float*>(forces);
    for (int64_t i = 0; i < natoms; ++i) {
      std::fprintf(f, "%d %d", ids ? ids[i] : static_cast<int32_t>(i + 1), types[i]);
      for (int a = 0; a < 3; ++a) {
        std::fputc(' ', f);
        put17(f, positions[3 * i + a]);
      }
      for (int a = 0; a < 3; ++a) {
        std::fputc(' ', f);
        put17(f, force_precision == TDMD_FP64 ? f64[3 * i + a]
                                              : static_cast<double>(f32[3 * i + a]));
      }
      std::fputc('\n', f);
    }
    out.close();
  });
}

int32_t tdmd_write_setfl(const char* path, const tdmd_eam* eam, const char* comment,
                         const double* masses, const char* elements) {
  return guarded([&] {
    TDMD_REQUIRE(path && eam, "null argument");
    TDMD_REQUIRE(eam->ntypes > 0 && !eam->F.empty(), "EAM tables are empty");
    const int nt = eam->ntypes;
    File out(path);
    std::FILE* f = out.f;
    if (!eam->comments.empty() && !comment) {
      for (const std::string& c : eam->comments) std::fprintf(f, "%s\n", c.c_str());
    } else {
      std::fprintf(f, "# %s\n# written by tdmd_write_setfl\n#\n", comment ? comment : "EAM");
    }
    std::vector<std::string> names = eam->elements;
    if (elements) {
      names.clear();
      std::istringstream is(elements);
      for (std::string w; is >> w;) names.push_back(w);
      TDMD_REQUIRE(static_cast<int>(names.size()) == nt, "one element name per type");
    }
    std::fprintf(f, "%d", nt);
    for (int t = 0; t < nt; ++t) {
      const bool have = t < static_cast<int>(names.size()) && !names[t].empty();
      std::fprintf(f, " %s", have ? names[t].c_str() : ("T" + std::to_string(t + 1)).c_str());
    }
    std::fputc('\n', f);
    std::fprintf(f, "%d ", eam->nrho);
    put17(f, eam->drho);
    std::fprintf(f, " %d ", eam->nr);
    put17(f, eam->dr);
    std::fputc(' ', f);
    put17(f, eam->cutoff);
    std::fputc('\n', f);
    auto block = [&](const double* v, int n) {
      for (int k = 0; k < n; ++k) {
        put17(f, v[k]);
        std::fputc((k % 5 == 4 || k == n - 1) ? '\n' : ' ', f);
      }
    };
    for (int t = 0; t < nt; ++t) {
      if (!masses && t < static_cast<int>(eam->headers.size()) && !eam->headers[t].empty()) {
        std::fprintf(f, "%s\n", eam->headers[t].c_str());
      } else {
        std::fprintf(f, "%d ", t + 1);
        put17(f, masses ? masses[t] : 1.0);
        std::fprintf(f, " 0.0 fcc\n");
      }
      block(eam->F.data() + static_cast<size_t>(t) * eam->nrho, eam->nrho);
      block(eam->rho.data() + static_cast<size_t>(t) * eam->nr, eam->nr);
    }
    const int npairs = nt * (nt + 1) / 2;
    for (int p = 0; p < npairs; ++p) block(eam->rphi.data() + static_cast<size_t>(p) * eam->nr,
                                           eam->nr);
    out.close();
  });
}

}  // extern "C"
