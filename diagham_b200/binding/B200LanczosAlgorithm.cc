// DiagHam-side binding of libdiagham_b200's Lanczos (see B200LanczosAlgorithm.h).
#include "B200LanczosAlgorithm.h"
#include "B200ParticleOnSphereHamiltonian.h"

#include <iostream>

using std::cout;
using std::endl;

B200LanczosAlgorithm::B200LanczosAlgorithm(AbstractArchitecture* architecture, int nbrEigenvalue, int maxIter,
					   int blockSize)
{
  this->Architecture = architecture;
  this->Hamiltonian = 0;
  this->Engine = 0;
  this->NbrEigenvalue = nbrEigenvalue;
  this->BlockSize = blockSize;
  // BasicLanczosAlgorithmWithGroundState converges one eigenvalue; more take the basic algorithm's
  // test on the nbrEigenvalue-th Ritz value (the engine forms Ritz vectors for either)
  if (blockSize > 1)
    this->Algorithm = DH_LANCZOS_BLOCK;
  else
    this->Algorithm = (nbrEigenvalue > 1) ? DH_LANCZOS_BASIC : DH_LANCZOS_WITH_GROUND_STATE;
  this->MaximumNumberIteration = maxIter;
  this->Dimension = 0;
  this->Eigenstates = 0;
  this->EigenvaluePrecision = MACHINE_PRECISION;
  this->EigenvectorPrecision = 0.0;
}

B200LanczosAlgorithm::~B200LanczosAlgorithm()
{
  delete[] this->Eigenstates;
  if (this->Engine != 0)
    dh_lanczos_destroy(this->Engine);
}

bool B200LanczosAlgorithm::Check(int status)
{
  if (status == DH_OK)
    return true;
  cout << "B200LanczosAlgorithm: " << dh_last_error() << endl;
  return false;
}

bool B200LanczosAlgorithm::IsReady()
{
  return this->Engine != 0;
}

void B200LanczosAlgorithm::SetHamiltonian(AbstractHamiltonian* hamiltonian)
{
  this->Hamiltonian = hamiltonian;
  if (this->Engine != 0)
    {
      dh_lanczos_destroy(this->Engine);
      this->Engine = 0;
    }
  B200ParticleOnSphereHamiltonian* H = dynamic_cast<B200ParticleOnSphereHamiltonian*>(hamiltonian);
  if ((H == 0) || (H->GetEngine() == 0))
    {
      cout << "B200LanczosAlgorithm: the Hamiltonian is not a B200ParticleOnSphereHamiltonian" << endl;
      return;
    }
  int64_t Dim = 0;
  dh_hamiltonian_get_dimension(H->GetEngine(), &Dim);
  this->Dimension = (long) Dim;
  dh_lanczos_t L = 0;
  if (!this->Check(dh_lanczos_create(H->GetEngine(), this->Algorithm, this->NbrEigenvalue, this->BlockSize,
				     this->MaximumNumberIteration, &L)))
    return;
  this->Engine = L;
  this->Check(dh_lanczos_set_eigenvalue_precision(this->Engine, this->EigenvaluePrecision));
}

void B200LanczosAlgorithm::SetEigenvaluePrecision(double precision)
{
  this->EigenvaluePrecision = precision;
  if (this->Engine != 0)
    this->Check(dh_lanczos_set_eigenvalue_precision(this->Engine, precision));
}

void B200LanczosAlgorithm::InitializeLanczosAlgorithm()
{
  if (this->Engine != 0)
    this->Check(dh_lanczos_initialize_random(this->Engine, 0));
}

void B200LanczosAlgorithm::InitializeLanczosAlgorithm(const Vector& vector)
{
  if (this->Engine != 0)
    this->Check(dh_lanczos_initialize(this->Engine, &((RealVector&) vector)[0], 1));
}

void B200LanczosAlgorithm::InitializeLanczosAlgorithm(Vector* vectors, int nbrVectors)
{
  if ((this->Engine == 0) || (nbrVectors <= 0))
    return;
  RealVector* V = (RealVector*) vectors;
  double* Block = new double[(long) nbrVectors * this->Dimension];
  for (int k = 0; k < nbrVectors; ++k)
    for (long i = 0; i < this->Dimension; ++i)
      Block[k * this->Dimension + i] = V[k][i];
  this->Check(dh_lanczos_initialize(this->Engine, Block, nbrVectors));
  delete[] Block;
}

void B200LanczosAlgorithm::RunLanczosAlgorithm(int nbrIter)
{
  if (this->Engine != 0)
    this->Check(dh_lanczos_run(this->Engine, nbrIter));
}

bool B200LanczosAlgorithm::TestConvergence()
{
  int Converged = 0;
  if ((this->Engine == 0) || !this->Check(dh_lanczos_test_convergence(this->Engine, &Converged)))
    return false;
  return Converged != 0;
}

RealTriDiagonalSymmetricMatrix& B200LanczosAlgorithm::GetDiagonalizedMatrix()
{
  int64_t Products = 0;
  int Rows = 0;
  if ((this->Engine == 0) || !this->Check(dh_lanczos_get_counters(this->Engine, &Products, &Rows)) || (Rows <= 0))
    return this->DiagonalizedMatrix;
  double* Values = new double[Rows];
  if (this->Check(dh_lanczos_get_eigenvalues(this->Engine, Values, Rows)))
    {
      this->DiagonalizedMatrix = RealTriDiagonalSymmetricMatrix(Rows, true);
      for (int i = 0; i < Rows; ++i)
	this->DiagonalizedMatrix.DiagonalElement(i) = Values[i];
    }
  delete[] Values;
  return this->DiagonalizedMatrix;
}

double B200LanczosAlgorithm::GetGroundStateEnergy()
{
  double E = 0.0;
  if (this->Engine != 0)
    this->Check(dh_lanczos_get_ground_state_energy(this->Engine, &E));
  this->GroundStateEnergy = E;
  return E;
}

Vector& B200LanczosAlgorithm::GetGroundState()
{
  this->GroundState = RealVector(this->Dimension, true);
  if (this->Engine != 0)
    this->Check(dh_lanczos_get_ground_state(this->Engine, &this->GroundState[0]));
  return this->GroundState;
}

Vector* B200LanczosAlgorithm::GetEigenstates(int nbrEigenstates)
{
  delete[] this->Eigenstates;
  this->Eigenstates = new RealVector[nbrEigenstates];
  double* All = new double[(long) nbrEigenstates * this->Dimension];
  if ((this->Engine != 0) && this->Check(dh_lanczos_get_eigenstates(this->Engine, nbrEigenstates, All)))
    for (int k = 0; k < nbrEigenstates; ++k)
      {
	this->Eigenstates[k] = RealVector(this->Dimension);
	for (long i = 0; i < this->Dimension; ++i)
	  this->Eigenstates[k][i] = All[k * this->Dimension + i];
      }
  delete[] All;
  return this->Eigenstates;
}
