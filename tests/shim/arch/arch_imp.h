// Stand-in for MISA-MD's arch/arch_imp.h, for compiling the misa_b200 hook shim in
// tests (the MISA-MD host is not part of this repository).
//
// It declares plain-data mirrors of the host types the shim reads, with the member
// names the reference plugin uses (src/hip_arch_acc_imp.cpp:47-150,
// src/memory/device_atoms.h:39-42), the Taywee/args pieces of src/cli.cpp:16-27, and the
// hook prototypes.  The potential mirror follows the host's interpolation tables: per
// atom type an electron-density and an embedding-energy table and per type pair a pair
// table holding r * phi(r), each a uniform grid {n, x0, invDx, values}.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

typedef int64_t _type_atom_count;
typedef int64_t _type_atom_index;
typedef int64_t NeiOffset;
typedef NeiOffset _type_neighbour_index_ele;

// ------------------------------------------------------------------ lattice atoms
struct AtomElement {
  long id;
  int type;
  double x[3];
  double v[3];
  double f[3];
  double rho;
  double df;
};

struct _type_atom_list_collection {
  AtomElement *atoms; // AoS layout (MD_ATOM_HASH_ARRAY_MEMORY_LAYOUT_AOS)
};

// ------------------------------------------------------------------------ domain
struct Region {
  int64_t x_low, y_low, z_low, x_high, y_high, z_high;
};

namespace comm {
struct BccDomain {
  Region dbx_sub_box_lattice_region;       // local box, doubled-x lattice indices
  int64_t dbx_sub_box_lattice_size[3];
  Region dbx_ghost_ext_lattice_region;     // box + ghost
  int64_t dbx_ghost_extended_lattice_size[3];
};
} // namespace comm

// ---------------------------------------------------------------- neighbour offsets
template <class T> struct NeighbourIndex {
  std::vector<T> nei_odd_offsets, nei_even_offsets;
  std::vector<T> nei_half_odd_offsets, nei_half_even_offsets;
};

// --------------------------------------------------------------------- potential
struct InterpolationObject {
  int n;
  double x0;
  double invDx;
  double *values;
};

struct OneWayEamList {
  std::vector<InterpolationObject> items; // index: atom type
  InterpolationObject *getEamItemByType(int type) {
    return type >= 0 && type < (int)items.size() ? &items[type] : nullptr;
  }
};

struct TwoWayEamList {
  int n_types = 0;
  std::vector<InterpolationObject> items; // (a, b) with a <= b, row-major upper triangle
  InterpolationObject *getPhiByEamPhiByType(int a, int b) {
    if (a > b) std::swap(a, b);
    if (a < 0 || b >= n_types) return nullptr;
    return &items[a * n_types - a * (a - 1) / 2 + (b - a)];
  }
};

struct eam {
  OneWayEamList electron_density; // f_t(r)
  OneWayEamList embedded;         // F_t(rho)
  TwoWayEamList eam_phi;          // r * phi_ab(r)
};

// ------------------------------------------------------------ Taywee/args pieces
namespace args {
struct ArgumentParser {
  std::vector<std::string> argv; // "-b", "4", ...
};
template <class T> struct ValueFlag {
  bool matched = false;
  T value{};
  ValueFlag(ArgumentParser &p, const std::string &, const std::string &, std::pair<char, std::string> names) {
    const std::string short_name = std::string("-") + names.first, long_name = "--" + names.second;
    for (size_t i = 0; i + 1 < p.argv.size(); i++)
      if (p.argv[i] == short_name || p.argv[i] == long_name) {
        matched = true;
        value = (T)std::stoul(p.argv[i + 1]);
      }
  }
  explicit operator bool() const { return matched; }
};
template <class T> T get(const ValueFlag<T> &f) { return f.value; }
} // namespace args

// ------------------------------------------------------------------------- hooks
void hip_env_init();
void hip_env_clean();
void hip_domain_init(const comm::BccDomain *p_domain);
void hip_nei_offset_init(const NeighbourIndex<_type_neighbour_index_ele> *nei_offset);
void hip_pot_init(eam *pot);
void hip_eam_rho_calc(eam *pot, _type_atom_list_collection atoms, double cutoff_radius);
void hip_eam_df_calc(eam *pot, _type_atom_list_collection atoms, double cutoff_radius);
void hip_eam_force_calc(eam *pot, _type_atom_list_collection atoms, double cutoff_radius);
bool hip_create_atoms_mem(void **atoms, std::size_t data_type_size, _type_atom_count size_x, _type_atom_count size_y,
                          _type_atom_count size_z);
bool hip_release_atoms_mem(void *atoms);
void hip_cli_options(args::ArgumentParser &parser);
bool hip_cli_options_parse(args::ArgumentParser &parser);
