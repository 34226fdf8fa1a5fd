// dropin_fqhe: the reference's own QHEOnSphereMainTask driven with the B200 binding in place.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile (target dropin) against the reference
// sources and linked with diagham_b200/libdiagham_b200.so and the DiagHam-side binding
// (diagham_b200/binding/).  It shows that an unmodified DiagHam driver runs on the GPU engine:
//
//   --engine reference   ParticleOnSphereGenericHamiltonian (ParticleOnSphereGenericHamiltonian.cc:66)
//   --engine b200        B200ParticleOnSphereHamiltonian (FP64 products on the GPU)
//   --engine b200-fp32   the same with FP32 matrix elements
//
// and, for the first two, hands the Hamiltonian to the unmodified QHEOnSphereMainTask
// (FQHE/src/MainTask/QHEOnSphereMainTask.cc) through MainTaskOperation, with the reference's own
// Lanczos classes chosen by the usual options (LanczosManager: --block-lanczos, --block-size,
// --iter-max, --nbr-eigen, --lanczos-precision, --initial-vector ...).  The task writes its spectrum
// file (one "Lz E" line per eigenvalue).
//
// --b200-lanczos instead runs B200LanczosAlgorithm (vectors in GPU memory) through the driver loop
// of QHEOnSphereMainTask.cc:732-753 (RunLanczosAlgorithm(nev + 2), then one step until
// TestConvergence or --iter-max) and writes the same spectrum lines.
#include "config.h"
#include "HilbertSpace/FermionOnSphere.h"
#include "Hamiltonian/ParticleOnSphereGenericHamiltonian.h"
#include "Architecture/ArchitectureManager.h"
#include "Architecture/AbstractArchitecture.h"
#include "Architecture/ArchitectureOperation/MainTaskOperation.h"
#include "LanczosAlgorithm/LanczosManager.h"
#include "MainTask/QHEOnSphereMainTask.h"
#include "Matrix/RealTriDiagonalSymmetricMatrix.h"
#include "Options/Options.h"

#include "B200ParticleOnSphereHamiltonian.h"
#include "B200LanczosAlgorithm.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>

using std::cout;
using std::endl;
using std::ofstream;

int main(int argc, char** argv)
{
  cout.precision(14);
  OptionManager Manager("dropin_fqhe", "0.01");
  ArchitectureManager Architecture;
  LanczosManager Lanczos(false);
  OptionGroup* SystemGroup = new OptionGroup("system options");
  OptionGroup* TaskGroup = new OptionGroup("main task options");
  Architecture.AddOptionGroup(&Manager);
  Lanczos.AddOptionGroup(&Manager);
  Manager += SystemGroup;
  Manager += TaskGroup;
  (*SystemGroup) += new SingleIntegerOption('p', "nbr-particles", "number of fermions", 8);
  (*SystemGroup) += new SingleIntegerOption('l', "lzmax", "twice the maximum momentum of a single particle", 21);
  (*SystemGroup) += new SingleIntegerOption('z', "twice-lz", "twice the total Lz of the sector", 0);
  (*SystemGroup) += new SingleStringOption('\n', "pseudopotentials",
					   "raw file of lzmax + 1 doubles V_0 .. V_lzmax (default: V_1 = 1)", 0);
  (*SystemGroup) += new SingleStringOption('\n', "engine", "reference, b200 or b200-fp32", "b200");
  (*SystemGroup) += new BooleanOption('\n', "b200-lanczos", "B200LanczosAlgorithm in the driver loop instead of the main task");
  (*SystemGroup) += new SingleStringOption('o', "output", "spectrum file", "spectrum.dat");
  // options the main task reads that the Lanczos and architecture groups do not declare
  (*TaskGroup) += new BooleanOption('\n', "get-lvalue", "compute the L value of each eigenstate");
  (*TaskGroup) += new BooleanOption('\n', "get-hvalue", "recompute <H> of each eigenstate");
  (*TaskGroup) += new BooleanOption('\n', "show-hamiltonian", "show the matrix of the Hamiltonian");
  (*TaskGroup) += new BooleanOption('\n', "test-hermitian", "test the hermiticity of the Hamiltonian");
  (*TaskGroup) += new BooleanOption('\n', "use-lapack", "use LAPACK for full diagonalisation");
  (*TaskGroup) += new BooleanOption('\n', "restart-projection", "projector option of the main task");
  (*TaskGroup) += new SingleDoubleOption('\n', "projector-precision", "projector option of the main task", 1e-14);
  (*TaskGroup) += new SingleIntegerOption('\n', "projector-iter-max", "projector option of the main task", 200);
  (*TaskGroup) += new SingleIntegerOption('\n', "projector-storage", "projector option of the main task", 1);
  (*TaskGroup) += new SingleStringOption('\n', "export-hamiltonian", "export the Hamiltonian to a file", 0);
  (*TaskGroup) += new SingleStringOption('\n', "save-precalculation", "save the precalculated elements", 0);
  (*TaskGroup) += new SingleStringOption('\n', "use-hilbert", "Hilbert subspace description", 0);
  if (Manager.ProceedOptions(argv, argc, cout) == false)
    {
      cout << "see man page for option syntax or type dropin_fqhe -h" << endl;
      return -1;
    }
  int N = Manager.GetInteger("nbr-particles");
  int LzMax = Manager.GetInteger("lzmax");
  int TwoLz = Manager.GetInteger("twice-lz");
  double* V = new double[LzMax + 1];
  for (int m = 0; m <= LzMax; ++m)
    V[m] = 0.0;
  if (Manager.GetString("pseudopotentials") != 0)
    {
      FILE* f = fopen(Manager.GetString("pseudopotentials"), "rb");
      if ((f == 0) || (fread(V, sizeof(double), LzMax + 1, f) != (size_t) (LzMax + 1)))
	{
	  cout << "cannot read " << LzMax + 1 << " doubles from " << Manager.GetString("pseudopotentials") << endl;
	  return 2;
	}
      fclose(f);
    }
  else
    V[1] = 1.0;
  const char* Engine = Manager.GetString("engine");
  bool Reference = strcmp(Engine, "reference") == 0;
  bool Fp32 = strcmp(Engine, "b200-fp32") == 0;
  if (!Reference && !Fp32 && (strcmp(Engine, "b200") != 0))
    {
      cout << "unknown engine " << Engine << endl;
      return 2;
    }

  FermionOnSphere Space(N, TwoLz, LzMax, 9ul << 20);
  AbstractArchitecture* Arch = Architecture.GetArchitecture();
  Arch->SetDimension(Space.GetHilbertSpaceDimension());
  AbstractQHEOnSphereHamiltonian* Hamiltonian;
  if (Reference)
    Hamiltonian = new ParticleOnSphereGenericHamiltonian(&Space, N, LzMax, V, 0.0, Arch, 0, false, 0, false);
  else
    {
      B200ParticleOnSphereHamiltonian* B = new B200ParticleOnSphereHamiltonian(&Space, N, LzMax, TwoLz, V, Arch, Fp32);
      if (!B->IsReady())
	{
	  cout << "the B200 engine could not be built: " << B->ErrorMessage() << endl;
	  return 3;
	}
      Hamiltonian = B;
    }
  char* Output = Manager.GetString("output");

  if (!Manager.GetBoolean("b200-lanczos"))
    {
      QHEOnSphereMainTask Task(&Manager, &Space, Hamiltonian, TwoLz, 0.0, Output, true, 0, LzMax);
      MainTaskOperation TaskOperation(&Task);
      TaskOperation.ApplyOperation(Arch);
    }
  else
    {
      if (Reference)
	{
	  cout << "--b200-lanczos needs a B200 engine" << endl;
	  return 2;
	}
      int NbrEigenvalue = Manager.GetInteger("nbr-eigen");
      int MaxIter = Manager.GetInteger("iter-max");
      int BlockSize = Manager.GetBoolean("block-lanczos") ? Manager.GetInteger("block-size") : 1;
      B200LanczosAlgorithm Algorithm(Arch, NbrEigenvalue, MaxIter, BlockSize);
      Algorithm.SetHamiltonian(Hamiltonian);
      if (!Algorithm.IsReady())
	return 3;
      if (Manager.GetDouble("lanczos-precision") != 0.0)
	Algorithm.SetEigenvaluePrecision(Manager.GetDouble("lanczos-precision"));
      Algorithm.InitializeLanczosAlgorithm();
      // the driver loop: nev + 2 steps first, then one at a time (counter in vectors)
      Algorithm.RunLanczosAlgorithm(NbrEigenvalue + 2);
      int Count = (NbrEigenvalue + 3) * BlockSize;
      while ((Algorithm.TestConvergence() == false) && (Count < MaxIter))
	{
	  Count += BlockSize;
	  Algorithm.RunLanczosAlgorithm(1);
	}
      RealTriDiagonalSymmetricMatrix Ritz;
      Ritz.Copy(Algorithm.GetDiagonalizedMatrix());
      Ritz.SortMatrixUpOrder();
      ofstream File;
      File.open(Output, std::ios::binary | std::ios::out);
      File.precision(14);
      for (int i = 0; (i < NbrEigenvalue) && (i < Ritz.GetNbrRow()); ++i)
	File << (TwoLz / 2) << " " << Ritz.DiagonalElement(i) << endl;
      File.close();
      cout << "B200LanczosAlgorithm: " << Count << " iterations, converged " << (Algorithm.TestConvergence() ? 1 : 0)
	   << ", E0 = " << Algorithm.GetGroundStateEnergy() << endl;
      RealVector& Psi = (RealVector&) Algorithm.GetGroundState();
      RealVector HPsi(Psi.GetVectorDimension(), true);
      Hamiltonian->LowLevelMultiply(Psi, HPsi);
      cout << "<psi|psi> = " << (Psi * Psi) << ", <psi|H|psi> = " << (Psi * HPsi) << endl;
    }
  delete Hamiltonian;
  delete[] V;
  return 0;
}
