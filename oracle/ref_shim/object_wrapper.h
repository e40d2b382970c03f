// Minimal stand-in for the reference's object_wrapper.h, used only when the
// reference's own hot-path sources are compiled as the parity oracle
// (oracle/build_ref.sh).  It provides the two things those sources touch:
// particle species metadata (name, mass, charge, sparsity settings, as
// particle_species.h names them) and the Parameters struct members read on
// the acceleration path.
#pragma once
#include <string>
#include <vector>
#include "definitions.h"

namespace species {
struct Species {
   std::string name{"proton"};
   Real charge{1.602176634e-19};
   Real mass{1.67262192e-27};
   Real sparseMinValue{1e-15};
   int sparseBlockAddWidthV{1};
   bool sparse_conserve_mass{false};
   int sparseDynamicAlgorithm{0};
   Real sparseDynamicBulkValue1{0};
   Real sparseDynamicBulkValue2{0};
   Real sparseDynamicMinValue1{0};
   Real sparseDynamicMinValue2{0};
};
}  // namespace species

struct ObjectWrapper {
   std::vector<species::Species> particleSpecies;
};
ObjectWrapper& getObjectWrapper();

struct Parameters {
   static uint bailout_velocity_space_wall_margin;
   static Real maxSlAccelerationRotation;
   static Real hallMinimumRhoq;
   static uint ohmGradPeTerm;
   static bool prepareForRebalance;
   static uint tstep;
   static bool vlasovAccelerateMaxwellianBoundaries;
};
typedef Parameters P;
