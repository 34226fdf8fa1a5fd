// DiagHam-side binding of libdiagham_b200's Lanczos: an AbstractLanczosAlgorithm
// (src/LanczosAlgorithm/AbstractLanczosAlgorithm.h:45-183) whose vectors stay in GPU memory.
//
// It stands where a driver builds BasicLanczosAlgorithm, BasicLanczosAlgorithmWithGroundState or
// BasicBlockLanczosAlgorithm (FQHE/src/MainTask/QHEOnSphereMainTask.cc:560-660) and keeps their
// interface: SetHamiltonian, InitializeLanczosAlgorithm, RunLanczosAlgorithm, TestConvergence,
// GetDiagonalizedMatrix, GetGroundState, GetEigenstates.  The Hamiltonian must be a
// B200ParticleOnSphereHamiltonian (its engine runs the products).  Compiled against the DiagHam
// headers (oracle/Makefile, target dropin); not part of libdiagham_b200.so.
#ifndef B200LANCZOSALGORITHM_H
#define B200LANCZOSALGORITHM_H

#include "config.h"
#include "LanczosAlgorithm/AbstractLanczosAlgorithm.h"
#include "Matrix/RealTriDiagonalSymmetricMatrix.h"
#include "Vector/RealVector.h"

#include "diagham_b200.h"

class B200LanczosAlgorithm : public AbstractLanczosAlgorithm
{
 protected:
  dh_lanczos_t Engine;
  int Algorithm;
  int NbrEigenvalue;
  int BlockSize;
  int MaximumNumberIteration;
  long Dimension;
  RealVector GroundState;
  RealVector* Eigenstates;

 public:
  // architecture = the driver's architecture; nbrEigenvalue, maxIter (in vectors, as --iter-max);
  // blockSize = 1 (BasicLanczosAlgorithmWithGroundState semantics for one eigenvalue,
  // BasicLanczosAlgorithm's for more) or 2, 4 (BasicBlockLanczosAlgorithm)
  B200LanczosAlgorithm(AbstractArchitecture* architecture, int nbrEigenvalue, int maxIter, int blockSize = 1);
  ~B200LanczosAlgorithm();

  // builds the engine on the Hamiltonian's GPU handle (a B200ParticleOnSphereHamiltonian)
  void SetHamiltonian(AbstractHamiltonian* hamiltonian);
  void SetEigenvaluePrecision(double precision);
  void InitializeLanczosAlgorithm();
  void InitializeLanczosAlgorithm(const Vector& vector);
  void InitializeLanczosAlgorithm(Vector* vectors, int nbrVectors);
  void RunLanczosAlgorithm(int nbrIter);
  bool TestConvergence();
  // the Ritz values on the diagonal (the driver sorts and prints them, QHEOnSphereMainTask.cc:754)
  RealTriDiagonalSymmetricMatrix& GetDiagonalizedMatrix();
  double GetGroundStateEnergy();
  Vector& GetGroundState();
  Vector* GetEigenstates(int nbrEigenstates);
  // false once a call into the engine failed (the message is printed)
  bool IsReady();

 protected:
  bool Check(int status);
};

#endif
