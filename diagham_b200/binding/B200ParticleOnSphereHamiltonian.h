// DiagHam-side binding of libdiagham_b200: a two-body Hamiltonian on FermionOnSphere whose products
// run on the GPU.
//
// It stands where a DiagHam program builds ParticleOnSphereGenericHamiltonian
// (FQHE/src/Programs/FQHEOnSphere/FQHESphereFermionsTwoBodyGeneric.cc:306) and is used through the
// AbstractHamiltonian interface (src/Hamiltonian/AbstractHamiltonian.h:228-344): the unmodified
// QHEOnSphereMainTask and Lanczos classes call LowLevelMultiply / LowLevelAddMultiply /
// LowLevelMultipleAddMultiply, which forward to the C ABI of include/diagham_b200.h with the
// RealVector storage (&v[0], src/Vector/RealVector.h:858) as host pointers.  Compiled against the
// DiagHam headers (oracle/Makefile, target dropin); not part of libdiagham_b200.so.
#ifndef B200PARTICLEONSPHEREHAMILTONIAN_H
#define B200PARTICLEONSPHEREHAMILTONIAN_H

#include "config.h"
#include "Hamiltonian/AbstractQHEOnSphereHamiltonian.h"
#include "HilbertSpace/FermionOnSphere.h"
#include "Vector/RealVector.h"

#include "diagham_b200.h"

class B200ParticleOnSphereHamiltonian : public AbstractQHEOnSphereHamiltonian
{
 protected:
  dh_space_t Space;
  dh_hamiltonian_t Engine;
  // the block that LowLevelMultipleAddMultiply hands to the engine ([row][k], k <= 4)
  double* BlockBuffer;
  long BlockCapacity;

 public:
  // particles = the reference's FermionOnSphere (the same sector is built on the GPU; the reference
  //             object stays the program's Hilbert space), nbrParticles, lzmax, totalLz = twice
  //             the sector's Lz; pseudoPotential = V_0 .. V_lzmax as for ParticleOnSphereGenericHamiltonian;
  // architecture = the program's architecture (products run as one GPU call per product);
  // fp32 = FP32 matrix elements with FP32 row accumulation (FP64 vectors)
  B200ParticleOnSphereHamiltonian(FermionOnSphere* particles, int nbrParticles, int lzmax, int totalLz,
				  double* pseudoPotential, AbstractArchitecture* architecture, bool fp32 = false);
  ~B200ParticleOnSphereHamiltonian();

  // true when the engine was built (false: ErrorMessage() says why)
  bool IsReady();
  const char* ErrorMessage();
  // the engine handle, for B200LanczosAlgorithm
  dh_hamiltonian_t GetEngine();

  void ShiftHamiltonian(double shift);
  // the GPU computes the whole product in one call: the SMP split of VectorHamiltonianMultiplyOperation
  // falls back to RawApplyOperation (VectorHamiltonianMultiplyOperation.cc:243-247)
  bool IsHamiltonianVectorOperationCompatible();
  bool IsHermitian();

  RealVector& LowLevelAddMultiply(RealVector& vSource, RealVector& vDestination, int firstComponent,
				  int nbrComponent);
  RealVector* LowLevelMultipleAddMultiply(RealVector* vSources, RealVector* vDestinations, int nbrVectors,
					  int firstComponent, int nbrComponent);

 protected:
  // the interaction factors live in the engine
  void EvaluateInteractionFactors();
};

#endif
