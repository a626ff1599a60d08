// MISA-MD architecture hooks backed by misa_b200.
//
// This file is the plugin side a MISA-MD build compiles in place of misa-md-hip's
// src/hip_arch_acc_imp.cpp, src/mem.cpp, src/cli.cpp and src/kernel_wrapper.hip.cpp:
// every hook MISA-MD's arch/arch_imp.h declares, with the reference's names and
// argument types, routed to the C ABI of include/misa_b200.h.  Build it inside MISA-MD
// with -I<this repository>/include and link misa-md-hip_b200/libmisa_b200.so.
//
// Host types used (all from the MISA-MD host, which declares them through
// arch/arch_imp.h):
//   comm::BccDomain            the fields hip_domain_init reads (hip_arch_acc_imp.cpp:47-76)
//   NeighbourIndex<T>          nei_{even,odd}_offsets and nei_half_{even,odd}_offsets
//   eam                        the host's tabulated potential (see table access below)
//   _type_atom_list_collection the lattice atom array (AoS: .atoms, 104-byte records)
//   args::ArgumentParser, args::ValueFlag  (Taywee/args, for -b/--batches)
//
// Errors: every misa_b200 call returns a status code; the hooks turn a failure into a
// std::runtime_error carrying mb_last_error(), where the reference aborts through
// HIP_CHECK.
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <vector_types.h> // dim3 (the CUDA runtime's)

#include "arch/arch_imp.h"
#include "misa_b200.h"

#ifdef MD_ATOM_HASH_ARRAY_MEMORY_LAYOUT_SOA
#error "misa_b200 hooks take the AoS lattice array (MD_ATOM_HASH_ARRAY_MEMORY_LAYOUT_AOS); the reference's SoA passes are empty too (src/double-buffer/rho_double_buffer_imp.cpp:63-68)"
#endif

namespace {

void ok(int rc, const char *what) {
  if (rc != MB_OK) throw std::runtime_error(std::string(what) + ": " + mb_last_error());
}

mb_atom_element *aos(_type_atom_list_collection atoms) {
  static_assert(sizeof(*atoms.atoms) == sizeof(mb_atom_element), "AtomElement must be the 104-byte record");
  return reinterpret_cast<mb_atom_element *>(atoms.atoms);
}

// ---------------------------------------------------------------- potential tables
// The reference hands `eam` to hip-potential (src/hip_arch_acc_imp.cpp:146-150), which
// copies the host's interpolation tables of types {0, 1, 2} to the device.  Here the
// knot values are read out of the same host tables: for each type t its electron
// density f_t(r) and embedding energy F_t(rho), for each pair (a, b) its pair term, all
// on uniform knots starting at x0 = 0 with spacing 1 / invDx.
//
// Pair convention: setfl files, and MISA-MD's tables read from them, hold r * phi(r);
// misa_b200 takes phi(r).  The knot values are divided by r_k (the r = 0 knot copies
// the first interior one: pairs never get that close).
struct HostTables {
  int n_types = 0, nr = 0, nrho = 0;
  double dr = 0, drho = 0, rmax = 0;
  std::vector<double> f, F, phi;
};

int pair_row(int a, int b, int n) {
  if (a > b) std::swap(a, b);
  return a * n - a * (a - 1) / 2 + (b - a);
}

template <class Item> void check_grid(const Item *it, const char *what) {
  if (!it || it->n < 2 || !(it->invDx > 0) || it->x0 != 0.0)
    throw std::runtime_error(std::string("hip_pot_init: ") + what +
                             " table must have >= 2 knots on a uniform grid starting at 0");
}

HostTables tables_from_eam(eam *pot) {
  HostTables h;
  // types 0, 1, 2 as the reference uploads them, as far as the host has tables for
  for (int t = 0; t < 3; t++) {
    if (!pot->electron_density.getEamItemByType(t) || !pot->embedded.getEamItemByType(t)) break;
    h.n_types = t + 1;
  }
  if (h.n_types == 0) throw std::runtime_error("hip_pot_init: the potential has no table for atom type 0");
  const auto *f0 = pot->electron_density.getEamItemByType(0);
  const auto *F0 = pot->embedded.getEamItemByType(0);
  check_grid(f0, "electron density");
  check_grid(F0, "embedding energy");
  h.nr = f0->n;
  h.nrho = F0->n;
  h.dr = 1.0 / f0->invDx;
  h.drho = 1.0 / F0->invDx;
  h.rmax = h.dr * (h.nr - 1);
  const int nt = h.n_types, np = nt * (nt + 1) / 2;
  h.f.assign((size_t)nt * h.nr, 0.0);
  h.F.assign((size_t)nt * h.nrho, 0.0);
  h.phi.assign((size_t)np * h.nr, 0.0);
  for (int t = 0; t < nt; t++) {
    const auto *ft = pot->electron_density.getEamItemByType(t);
    const auto *Ft = pot->embedded.getEamItemByType(t);
    check_grid(ft, "electron density");
    check_grid(Ft, "embedding energy");
    if (ft->n != h.nr || Ft->n != h.nrho || ft->invDx != f0->invDx || Ft->invDx != F0->invDx)
      throw std::runtime_error("hip_pot_init: every type's tables must share one r grid and one rho grid");
    for (int k = 0; k < h.nr; k++) h.f[(size_t)t * h.nr + k] = ft->values[k];
    for (int k = 0; k < h.nrho; k++) h.F[(size_t)t * h.nrho + k] = Ft->values[k];
  }
  for (int a = 0; a < nt; a++)
    for (int b = a; b < nt; b++) {
      const auto *pt = pot->eam_phi.getPhiByEamPhiByType(a, b);
      check_grid(pt, "pair");
      if (pt->n != h.nr || pt->invDx != f0->invDx)
        throw std::runtime_error("hip_pot_init: pair tables must share the electron density's r grid");
      double *row = h.phi.data() + (size_t)pair_row(a, b, nt) * h.nr;
      for (int k = 1; k < h.nr; k++) row[k] = pt->values[k] / (k * h.dr); // r * phi -> phi
      row[0] = row[1];
    }
  return h;
}

unsigned int g_batches = 1;

} // namespace

// ------------------------------------------------------ src/hip_arch_acc_imp.cpp:28-225

void hip_env_init() { ok(mb_env_init(0), "hip_env_init"); } // device 0, as the reference (:31)

void hip_env_clean() { ok(mb_env_clean(), "hip_env_clean"); }

void hip_domain_init(const comm::BccDomain *p_domain) {
  mb_device_domain d{};
  d.ghost_size_x = p_domain->dbx_sub_box_lattice_region.x_low - p_domain->dbx_ghost_ext_lattice_region.x_low;
  d.ghost_size_y = p_domain->dbx_sub_box_lattice_region.y_low - p_domain->dbx_ghost_ext_lattice_region.y_low;
  d.ghost_size_z = p_domain->dbx_sub_box_lattice_region.z_low - p_domain->dbx_ghost_ext_lattice_region.z_low;
  d.box_size_x = p_domain->dbx_sub_box_lattice_size[0];
  d.box_size_y = p_domain->dbx_sub_box_lattice_size[1];
  d.box_size_z = p_domain->dbx_sub_box_lattice_size[2];
  d.ext_size_x = p_domain->dbx_ghost_extended_lattice_size[0];
  d.ext_size_y = p_domain->dbx_ghost_extended_lattice_size[1];
  d.ext_size_z = p_domain->dbx_ghost_extended_lattice_size[2];
  d.box_index_start_x = p_domain->dbx_sub_box_lattice_region.x_low;
  d.box_index_start_y = p_domain->dbx_sub_box_lattice_region.y_low;
  d.box_index_start_z = p_domain->dbx_sub_box_lattice_region.z_low;
  ok(mb_domain_init(&d), "hip_domain_init");
}

void hip_nei_offset_init(const NeighbourIndex<_type_neighbour_index_ele> *nei_offset) {
#ifndef USE_NEWTONS_THIRD_LOW
  const auto &ev = nei_offset->nei_even_offsets;
  const auto &od = nei_offset->nei_odd_offsets;
#else
  ok(mb_set_half_neighbour(1), "hip_nei_offset_init"); // :118-130, the half stencils
  const auto &ev = nei_offset->nei_half_even_offsets;
  const auto &od = nei_offset->nei_half_odd_offsets;
#endif
  std::vector<int64_t> even(ev.size()), odd(od.size());
  for (size_t i = 0; i < ev.size(); i++) even[i] = (int64_t)ev[i];
  for (size_t i = 0; i < od.size(); i++) odd[i] = (int64_t)od[i];
  ok(mb_nei_offset_init(even.data(), even.size(), odd.data(), odd.size()), "hip_nei_offset_init");
}

void hip_pot_init(eam *_pot) {
  HostTables h = tables_from_eam(_pot);
  mb_eam_tables t{};
  t.n_types = h.n_types;
  t.nr = h.nr;
  t.nrho = h.nrho;
  t.dr = h.dr;
  t.drho = h.drho;
  t.cutoff = h.rmax; // each pass takes its own cutoff radius from the hook call
  t.f = h.f.data();
  t.F = h.F.data();
  t.phi = h.phi.data();
  ok(mb_pot_init(&t), "hip_pot_init"); // builds and uploads its own spline tables from the knots
}

void hip_eam_rho_calc(eam *, _type_atom_list_collection _atoms, double cutoff_radius) {
  ok(mb_eam_rho_calc(aos(_atoms), cutoff_radius), "hip_eam_rho_calc");
}

void hip_eam_df_calc(eam *, _type_atom_list_collection _atoms, double cutoff_radius) {
  // full-neighbour build: returns at once (df came out of the rho pass, :184-186);
  // half-neighbour build: df = F'(rho) of the box sites
  ok(mb_eam_df_calc(aos(_atoms), cutoff_radius), "hip_eam_df_calc");
}

void hip_eam_force_calc(eam *, _type_atom_list_collection _atoms, double cutoff_radius) {
  ok(mb_eam_force_calc(aos(_atoms), cutoff_radius), "hip_eam_force_calc");
}

// ----------------------------------------------------------------- src/mem.cpp:14-32

bool hip_create_atoms_mem(void **atoms, std::size_t data_type_size, _type_atom_count size_x, _type_atom_count size_y,
                          _type_atom_count size_z) {
  int allocated = 0;
  ok(mb_create_atoms_mem(atoms, data_type_size, (int64_t)size_x, (int64_t)size_y, (int64_t)size_z, &allocated),
     "hip_create_atoms_mem");
  return allocated != 0;
}

bool hip_release_atoms_mem(void *atoms) {
  int released = 0;
  ok(mb_release_atoms_mem(atoms, &released), "hip_release_atoms_mem");
  return released != 0;
}

// ----------------------------------------------------------------- src/cli.cpp:16-27

namespace {
args::ValueFlag<unsigned int> *g_flag_batches = nullptr;
}

void hip_cli_options(args::ArgumentParser &parser) {
  g_flag_batches = new args::ValueFlag<unsigned int>(parser, "batches", "batches", {'b', "Batches number"});
}

bool hip_cli_options_parse(args::ArgumentParser &) {
  if (g_flag_batches && *g_flag_batches) {
    g_batches = args::get(*g_flag_batches);
    // z-slabs the rho and force hooks stream the array in; the results do not depend on it
    ok(mb_cli_set_batches(g_batches), "hip_cli_options_parse");
  }
  return true;
}

// ------------------------------------------------- src/kernel_wrapper.hip.cpp:9-22
// Legacy launchers, kept so that MISA-MD builds which still reference them link.  In
// the reference they launch kernels that compute nothing: calc_rho and calForce have
// empty bodies (src/kernels/hip_kernels.hip.cpp:19,45) and calDf is launched on the
// empty range [0, 0) (kernel_wrapper.hip.cpp:15-17).  They do nothing here either.

// The plugin's own record and stencil types, as the reference declares them
// (src/kernel_types.h:40-48, 66-71): the launchers' mangled names depend on them.
typedef struct {
  long id;
  int type;
  double x[3];
  double v[3];
  double f[3];
  double rho;
  double df;
} _cuAtomElement;
typedef struct {
  size_t nei_odd_size;
  size_t nei_even_size;
  NeiOffset *nei_odd;
  NeiOffset *nei_even;
} _hipDeviceNeiOffsets;
static_assert(sizeof(_cuAtomElement) == sizeof(mb_atom_element), "the record is 104 bytes");

void __kernel_calRho_wrapper(dim3, dim3, _cuAtomElement *, _hipDeviceNeiOffsets, double) {}
void __kernel_calDf_wrapper(dim3, dim3, _cuAtomElement *) {}
void __kernel_calForce_wrapper(dim3, dim3, _cuAtomElement *, _hipDeviceNeiOffsets, double) {}
