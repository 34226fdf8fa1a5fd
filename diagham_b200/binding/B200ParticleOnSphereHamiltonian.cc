// DiagHam-side binding of libdiagham_b200 (see B200ParticleOnSphereHamiltonian.h).
#include "B200ParticleOnSphereHamiltonian.h"

#include <cstring>
#include <iostream>

using std::cout;
using std::endl;

B200ParticleOnSphereHamiltonian::B200ParticleOnSphereHamiltonian(FermionOnSphere* particles, int nbrParticles,
								 int lzmax, int totalLz, double* pseudoPotential,
								 AbstractArchitecture* architecture, bool fp32)
{
  // the members the base classes read (AbstractQHEOnSphereHamiltonian.cc:58-109, :3547)
  this->Particles = particles;
  this->NbrParticles = nbrParticles;
  this->LzMax = lzmax;
  this->NbrLzValue = lzmax + 1;
  this->Architecture = architecture;
  this->HamiltonianShift = 0.0;
  this->L2Operator = 0;
  this->FastMultiplicationFlag = false;
  this->DiskStorageFlag = false;
  this->OneBodyTermFlag = false;
  this->InteractionFactors = 0;
  this->NbrInteractionFactors = 0;
  this->Space = 0;
  this->Engine = 0;
  this->BlockBuffer = 0;
  this->BlockCapacity = 0;
  if (dh_fermion_on_sphere_create(nbrParticles, totalLz, lzmax, 9ul << 20, &this->Space) != DH_OK ||
      dh_particle_on_sphere_generic_hamiltonian_create(this->Space, nbrParticles, lzmax, pseudoPotential, 0.0,
						       &this->Engine) != DH_OK)
    {
      cout << "B200ParticleOnSphereHamiltonian: " << dh_last_error() << endl;
      return;
    }
  int64_t Dim = 0;
  dh_hamiltonian_get_dimension(this->Engine, &Dim);
  if (Dim != (int64_t) particles->GetHilbertSpaceDimension())
    {
      cout << "B200ParticleOnSphereHamiltonian: the GPU sector has " << Dim << " states, the space "
	   << particles->GetHilbertSpaceDimension() << endl;
      dh_hamiltonian_destroy(this->Engine);
      this->Engine = 0;
      return;
    }
  if (fp32)
    dh_hamiltonian_set_precision(this->Engine, DH_PRECISION_FP32);
}

B200ParticleOnSphereHamiltonian::~B200ParticleOnSphereHamiltonian()
{
  delete[] this->BlockBuffer;
  if (this->Engine != 0)
    dh_hamiltonian_destroy(this->Engine);
  if (this->Space != 0)
    dh_space_destroy(this->Space);
}

bool B200ParticleOnSphereHamiltonian::IsReady()
{
  return this->Engine != 0;
}

const char* B200ParticleOnSphereHamiltonian::ErrorMessage()
{
  return dh_last_error();
}

dh_hamiltonian_t B200ParticleOnSphereHamiltonian::GetEngine()
{
  return this->Engine;
}

void B200ParticleOnSphereHamiltonian::EvaluateInteractionFactors()
{
}

void B200ParticleOnSphereHamiltonian::ShiftHamiltonian(double shift)
{
  this->HamiltonianShift = shift;
  if (this->Engine != 0)
    dh_hamiltonian_shift(this->Engine, shift);
}

bool B200ParticleOnSphereHamiltonian::IsHamiltonianVectorOperationCompatible()
{
  return false;
}

bool B200ParticleOnSphereHamiltonian::IsHermitian()
{
  return false;
}

RealVector& B200ParticleOnSphereHamiltonian::LowLevelAddMultiply(RealVector& vSource, RealVector& vDestination,
								  int firstComponent, int nbrComponent)
{
  if ((this->Engine == 0) || (nbrComponent <= 0))
    return vDestination;
  if (dh_hamiltonian_low_level_add_multiply(this->Engine, &vSource[0], &vDestination[0], firstComponent,
					    nbrComponent) != DH_OK)
    cout << "B200ParticleOnSphereHamiltonian: " << dh_last_error() << endl;
  return vDestination;
}

RealVector* B200ParticleOnSphereHamiltonian::LowLevelMultipleAddMultiply(RealVector* vSources,
									  RealVector* vDestinations, int nbrVectors,
									  int firstComponent, int nbrComponent)
{
  if ((this->Engine == 0) || (nbrComponent <= 0) || (nbrVectors <= 0))
    return vDestinations;
  // the engine takes the vectors one after the other: one call enumerates every row once for all
  // of them (AbstractQHEOnSphereHamiltonian.cc:1217 does the same per row on the CPU)
  long Dim = this->Particles->GetHilbertSpaceDimension();
  long Need = 2l * nbrVectors * Dim;
  if (Need > this->BlockCapacity)
    {
      delete[] this->BlockBuffer;
      this->BlockBuffer = new double[Need];
      this->BlockCapacity = Need;
    }
  double* Src = this->BlockBuffer;
  double* Dst = this->BlockBuffer + (long) nbrVectors * Dim;
  for (int k = 0; k < nbrVectors; ++k)
    {
      memcpy(Src + k * Dim, &vSources[k][0], Dim * sizeof(double));
      memcpy(Dst + k * Dim, &vDestinations[k][0], Dim * sizeof(double));
    }
  if (dh_hamiltonian_low_level_multiple_add_multiply(this->Engine, Src, Dst, nbrVectors, firstComponent,
						      nbrComponent) != DH_OK)
    {
      cout << "B200ParticleOnSphereHamiltonian: " << dh_last_error() << endl;
      return vDestinations;
    }
  for (int k = 0; k < nbrVectors; ++k)
    memcpy(&vDestinations[k][0], Dst + k * Dim, Dim * sizeof(double));
  return vDestinations;
}
