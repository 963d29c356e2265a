// Host-side mechanism model for the NRG chemistry step.
//
// Holds the constant tables that the reference builds at set-up time
// (chemical_properties_class.f90:117-181 and thermophysical_properties_class.f90:
// 137-210) and the derived per-reaction update lists the GPU kernels use.
#pragma once

#include <string>
#include <vector>

namespace nrg {

constexpr double kRGasJ = 8.31446261815324;    // global_data.f90:36
constexpr double kRGasCal = 1.98720425864083;  // global_data.f90:37
constexpr double kTRef = 298.15;               // global_data.f90:38
constexpr double kPAtm = 101325.0;             // global_data.f90:39
constexpr double kTCeiling = 6000.0;           // global_data.f90:44

enum class EactUnits { J_mol = 0, kJ_mol = 1, cal_mol = 2, kcal_mol = 3 };

struct Reaction {
  int type = 0;          // reference reactions_type (0..7)
  int n_left = 0, n_right = 0;
  int left[3] = {0, 0, 0};   // 1-based species, n+1 = M
  int right[3] = {0, 0, 0};
  double A = 0, beta = 0, E = 0;            // E in J/mol after unit conversion
  double A_low = 0, beta_low = 0, E_low = 0;
  double troe[4] = {0, 0, 0, 0};
};

struct Mechanism {
  std::vector<std::string> species;  // n species; "M" is index n (0-based)
  std::vector<Reaction> reactions;
  std::vector<double> eff;           // [r * n + k]
  std::vector<double> a_coeffs;      // [(k * 2 + set) * 7 + i], multiplied by R
  std::vector<double> molar_mass;    // kg/mol
  // transport deck (load_transport): eps/k_B [K], sigma [nm], binary
  // diffusivity constants [i * n + j] (symmetric, 0 on the diagonal)
  std::vector<double> well_depth, collision_diameter, binary_diffusivity;
  int n() const { return (int)species.size(); }
  int r() const { return (int)reactions.size(); }
};

// Parse the three reference input decks.  Returns an empty string on success
// or a message naming the failure (the reference stops the program instead).
std::string load_mechanism(const std::string& mech_path, const std::string& thermo_path,
                           const std::string& molar_path, double eff_default, EactUnits units,
                           Mechanism* out);

// Transport deck for the species of m (thermophysical_properties_class.f90:
// 1343-1414); empty string on success.
std::string load_transport(const std::string& transport_path, Mechanism* m);

// NASA-7 helpers with the reference's evaluation order
// (thermophysical_properties_class.f90:225-300).
double specie_enthalpy(const Mechanism& m, double T, int k);
double specie_entropy(const Mechanism& m, double T, int k);
double specie_cp(const Mechanism& m, double T, int k);

}  // namespace nrg
