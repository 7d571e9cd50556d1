// Host-side description of a synthetic plane-wave system (set-up data).
#pragma once

#include <array>
#include <cstdint>
#include <vector>

#include "chfsi.h"

namespace chfsi {

struct System {
    chfsi_synth_params params{};
    double a = 0.0, omega = 0.0, lattice[9] = {};
    int ngrid[3] = {0, 0, 0};
    int ngrid_density[3] = {0, 0, 0};
    double q_width = 0.0;
    int uspp = 0;
    int n_atoms = 0, n_occ = 0, n_bands = 0, n_pw = 0, n_columns = 0;
    int n_proj = 0, n_ions_proj = 0;
    double n_elec = 0.0, gmax = 0.0, e_ewald = 0.0;
    std::vector<double> pos, zion, occ;
    std::vector<int32_t> miller;        // n_pw x 3
    std::vector<double> kinetic;        // n_pw
    std::vector<double> vloc_g;         // 2 x ngrid^3 (interleaved complex)
    std::vector<double> beta;           // 2 x n_proj x n_pw
    std::vector<int32_t> proj_offsets;  // n_ions_proj + 1
    std::vector<double> dmat, qmat;     // 2 x sum ne_i^2
    std::vector<double> psi0;           // 2 x n_bands x n_pw
};

// pos_override: n_atoms x 3 Cartesian positions in place of the seeded lattice
chfsi_status generate_system(const chfsi_synth_params& p, System& s,
                             const double* pos_override = nullptr);
int next_smooth235(int n);

}  // namespace chfsi
