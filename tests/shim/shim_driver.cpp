// Test driver of the MISA-MD hook shim: builds the host-side objects a MISA-MD timestep
// holds (BccDomain, NeighbourIndex, eam, the AoS atom list) from plain arrays and calls
// the hooks by their reference names, so that tests/test_shim.py can drive them through
// ctypes.  Each entry point returns 0, or 1 with the hook's exception text in err.
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include "arch/arch_imp.h"

namespace {
eam g_pot;
std::vector<double> g_knots; // storage behind the InterpolationObject values

int caught(const std::exception &e, char *err, int cap) {
  if (err && cap > 0) std::snprintf(err, (size_t)cap, "%s", e.what());
  return 1;
}
} // namespace

extern "C" {

int drive_env_init(char *err, int cap) {
  try {
    hip_env_init();
  } catch (const std::exception &e) {
    return caught(e, err, cap);
  }
  return 0;
}

int drive_env_clean(char *err, int cap) {
  try {
    hip_env_clean();
  } catch (const std::exception &e) {
    return caught(e, err, cap);
  }
  return 0;
}

// -b <batches> through hip_cli_options / hip_cli_options_parse.
int drive_cli(const char *batches, char *err, int cap) {
  try {
    args::ArgumentParser p;
    if (batches) p.argv = {"md", "-b", batches};
    hip_cli_options(p);
    hip_cli_options_parse(p);
  } catch (const std::exception &e) {
    return caught(e, err, cap);
  }
  return 0;
}

// hip_domain_init of a box whose first local lattice index is (sx, sy, sz) (doubled x),
// hip_nei_offset_init of the full stencils, hip_pot_init of tables f [nt][nr],
// F [nt][nrho] and r * phi [nt (nt + 1) / 2][nr] on knots from 0.
int drive_setup(const int64_t box[3], const int64_t ghost[3], const int64_t start[3], const int64_t *even,
                int n_even, const int64_t *odd, int n_odd, int n_types, int nr, double dr, int nrho, double drho,
                const double *f, const double *F, const double *rphi, char *err, int cap) {
  try {
    comm::BccDomain d{};
    d.dbx_sub_box_lattice_region = {start[0], start[1], start[2], start[0] + box[0], start[1] + box[1],
                                    start[2] + box[2]};
    d.dbx_ghost_ext_lattice_region = {start[0] - ghost[0], start[1] - ghost[1], start[2] - ghost[2],
                                      start[0] + box[0] + ghost[0], start[1] + box[1] + ghost[1],
                                      start[2] + box[2] + ghost[2]};
    for (int k = 0; k < 3; k++) {
      d.dbx_sub_box_lattice_size[k] = box[k];
      d.dbx_ghost_extended_lattice_size[k] = box[k] + 2 * ghost[k];
    }
    hip_domain_init(&d);
    NeighbourIndex<_type_neighbour_index_ele> n;
    n.nei_even_offsets.assign(even, even + n_even);
    n.nei_odd_offsets.assign(odd, odd + n_odd);
    hip_nei_offset_init(&n);
    const int np = n_types * (n_types + 1) / 2;
    g_knots.assign(f, f + (size_t)n_types * nr);
    g_knots.insert(g_knots.end(), F, F + (size_t)n_types * nrho);
    g_knots.insert(g_knots.end(), rphi, rphi + (size_t)np * nr);
    g_pot = eam();
    double *base = g_knots.data();
    for (int t = 0; t < n_types; t++)
      g_pot.electron_density.items.push_back({nr, 0.0, 1.0 / dr, base + (size_t)t * nr});
    base += (size_t)n_types * nr;
    for (int t = 0; t < n_types; t++) g_pot.embedded.items.push_back({nrho, 0.0, 1.0 / drho, base + (size_t)t * nrho});
    base += (size_t)n_types * nrho;
    g_pot.eam_phi.n_types = n_types;
    for (int q = 0; q < np; q++) g_pot.eam_phi.items.push_back({nr, 0.0, 1.0 / dr, base + (size_t)q * nr});
    hip_pot_init(&g_pot);
  } catch (const std::exception &e) {
    return caught(e, err, cap);
  }
  return 0;
}

// which: 0 rho, 1 df, 2 force, on the host's ghost-extended AoS array.
int drive_pass(int which, void *atoms, double cutoff, char *err, int cap) {
  try {
    _type_atom_list_collection c{static_cast<AtomElement *>(atoms)};
    if (which == 0) hip_eam_rho_calc(&g_pot, c, cutoff);
    if (which == 1) hip_eam_df_calc(&g_pot, c, cutoff);
    if (which == 2) hip_eam_force_calc(&g_pot, c, cutoff);
  } catch (const std::exception &e) {
    return caught(e, err, cap);
  }
  return 0;
}

// hip_create_atoms_mem / hip_release_atoms_mem round trip: page-locked host memory.
int drive_atoms_mem(int64_t x, int64_t y, int64_t z, int *created, int *released, char *err, int cap) {
  try {
    void *p = nullptr;
    *created = hip_create_atoms_mem(&p, sizeof(AtomElement), x, y, z) ? 1 : 0;
    std::memset(p, 0, (size_t)(x * y * z) * sizeof(AtomElement));
    *released = hip_release_atoms_mem(p) ? 1 : 0;
  } catch (const std::exception &e) {
    return caught(e, err, cap);
  }
  return 0;
}

} // extern "C"
