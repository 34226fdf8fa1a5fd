// ref_tool: a thin command-line driver over DiagHam's own classes.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled (by oracle/Makefile) against
// the reference sources and linked into oracle/_ref/ref_tool.  It is used to
// generate the golden fixtures under tests/golden/ and, in bench.py, to time the
// reference CPU implementation of the hot path.  No product code links it.
//
// Every command calls only reference classes:
//   FermionOnSphere                      FQHE/src/HilbertSpace/FermionOnSphere.cc:75
//   BosonOnSphereShort                   FQHE/src/HilbertSpace/BosonOnSphereShort.cc:81 (bqhe_* commands)
//   ParticleOnSphereGenericHamiltonian   FQHE/src/Hamiltonian/ParticleOnSphereGenericHamiltonian.cc:66
//   AbstractQHEOnSphereHamiltonian::LowLevelAddMultiply   .../AbstractQHEOnSphereHamiltonian.cc:410
//   Spin1_2Chain                         Spin/src/HilbertSpace/Spin1_2Chain.cc:113
//   BasicLanczosAlgorithm / FullReorthogonalizedLanczosAlgorithm / BasicBlockLanczosAlgorithm
//   BasicLanczosAlgorithmWithDiskStorage / BasicLanczosAlgorithmWithGroundStateDiskStorage
//   EvaluatePseudopotentials             FQHE/src/Tools/FQHESpectrum/PseudoPotentials.cc:35
//   VectorHamiltonianMultiplyOperation on SMPArchitecture (the reference SMP path)
//
// The J1-J2 chain on a plain Spin1_2Chain has no reference Hamiltonian class,
// so J1J2ChainHarness below applies the element pattern of
// SpinChainJ1J2RealHamiltonianWithTranslations.cc:94-192 / :335-352 through the
// API model of SpinChainHamiltonian.cc:257-298, calling the reference
// Spin1_2Chain::SmiSpj / SziSzj / FindStateIndex for every element.
//
// Binary outputs are little-endian raw arrays; tests/golden/make_golden.py
// documents each layout and converts them to .npz fixtures.

#include "config.h"
#include "HilbertSpace/FermionOnSphere.h"
#include "HilbertSpace/FermionOnSphereLong.h"
#include "HilbertSpace/BosonOnSphereShort.h"
#include "HilbertSpace/Spin1_2Chain.h"
#include "HilbertSpace/Spin1_2ChainWithTranslations.h"
#include "Hamiltonian/SpinChainJ1J2RealHamiltonianWithTranslations.h"
#include "Hamiltonian/SpinChainJ1J2HamiltonianWithTranslations.h"
#include "Vector/ComplexVector.h"
#include "Hamiltonian/ParticleOnSphereGenericHamiltonian.h"
#include "Hamiltonian/ParticleOnSphereL2Hamiltonian.h"
#include "Hamiltonian/AbstractHamiltonian.h"
#include "Architecture/MonoProcessorArchitecture.h"
#include "Architecture/SMPArchitecture.h"
#include "Architecture/ArchitectureOperation/VectorHamiltonianMultiplyOperation.h"
#include "Architecture/ArchitectureOperation/MultipleVectorHamiltonianMultiplyOperation.h"
#include "LanczosAlgorithm/BasicLanczosAlgorithm.h"
#include "LanczosAlgorithm/FullReorthogonalizedLanczosAlgorithm.h"
#include "LanczosAlgorithm/BasicBlockLanczosAlgorithm.h"
#include "LanczosAlgorithm/BasicLanczosAlgorithmWithGroundState.h"
#include "LanczosAlgorithm/BasicLanczosAlgorithmWithDiskStorage.h"
#include "LanczosAlgorithm/BasicLanczosAlgorithmWithGroundStateDiskStorage.h"
#include "Matrix/RealTriDiagonalSymmetricMatrix.h"
#include "Matrix/RealMatrix.h"
#include "Matrix/RealSymmetricMatrix.h"
#include "Tools/FQHESpectrum/PseudoPotentials.h"
#include "Vector/RealVector.h"
#include "MathTools/Complex.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>
#include <sys/time.h>
#include <unistd.h>
#include <iostream>
#include <string>
#include <sstream>

using std::cout;
using std::endl;

static double Now()
{
  timeval t;
  gettimeofday(&t, 0);
  return t.tv_sec + 1e-6 * t.tv_usec;
}

static FILE* OpenOut(const char* name)
{
  FILE* f = fopen(name, "wb");
  if (f == 0)
    {
      fprintf(stderr, "cannot open %s\n", name);
      exit(2);
    }
  return f;
}

// pseudopotentials are read from a raw file of (2S+1) doubles (V_0 .. V_2S)
static double* ReadDoubles(const char* name, long n)
{
  double* v = new double[n];
  FILE* f = fopen(name, "rb");
  if ((f == 0) || (fread(v, sizeof(double), n, f) != (size_t) n))
    {
      fprintf(stderr, "cannot read %ld doubles from %s\n", n, name);
      exit(2);
    }
  fclose(f);
  return v;
}

static int* ReadInts(const char* name, long& n)
{
  FILE* f = fopen(name, "rb");
  if (f == 0)
    {
      fprintf(stderr, "cannot read %s\n", name);
      exit(2);
    }
  fseek(f, 0, SEEK_END);
  n = ftell(f) / sizeof(int);
  fseek(f, 0, SEEK_SET);
  int* v = new int[n];
  if (fread(v, sizeof(int), n, f) != (size_t) n)
    exit(2);
  fclose(f);
  return v;
}

// exposes the protected basis arrays of the reference Hilbert spaces
class ExposedFermionOnSphere : public FermionOnSphere
{
 public:
  ExposedFermionOnSphere(int nbrFermions, int totalLz, int lzMax, unsigned long memory)
    : FermionOnSphere(nbrFermions, totalLz, lzMax, memory)
  {
  }
  unsigned long Word(long i) { return this->StateDescription[i]; }
  int WordLzMax(long i) { return this->StateLzMax[i]; }
  int Find(unsigned long w, int lzmax) { return this->FindStateIndex(w, lzmax); }
};

class ExposedFermionOnSphereLong : public FermionOnSphereLong
{
 public:
  ExposedFermionOnSphereLong(int nbrFermions, int totalLz, int lzMax, unsigned long memory)
    : FermionOnSphereLong(nbrFermions, totalLz, lzMax, memory)
  {
  }
  // the 128-bit word as its low and high 64-bit halves
  unsigned long WordLow(long i) { return (unsigned long) this->StateDescription[i]; }
  unsigned long WordHigh(long i) { return (unsigned long) (this->StateDescription[i] >> 64); }
};

class ExposedSpin1_2Chain : public Spin1_2Chain
{
 public:
  ExposedSpin1_2Chain(int chainLength, int sz, int memory) : Spin1_2Chain(chainLength, sz, memory)
  {
  }
  unsigned long Word(long i) { return this->StateDescription[i]; }
  int Find(unsigned long w) { return this->FindStateIndex(w); }
};

// exposes the protected interaction tables of the reference Hamiltonian
class ExposedGenericHamiltonian : public ParticleOnSphereGenericHamiltonian
{
 public:
  ExposedGenericHamiltonian(ParticleOnSphere* particles, int nbrParticles, int lzmax, double* pseudo,
			    AbstractArchitecture* arch, bool hermitian)
    : ParticleOnSphereGenericHamiltonian(particles, nbrParticles, lzmax, pseudo, 0.0, arch, 0, false, 0, hermitian)
  {
  }
  int GetNbrM12() { return this->NbrM12Indices; }
  int M1(int i) { return this->M1Value[i]; }
  int M2(int i) { return this->M2Value[i]; }
  int NbrM3(int i) { return this->NbrM3Values[i]; }
  int M3(int i, int j) { return this->M3Values[i][j]; }
  int NbrFactors() { return this->NbrInteractionFactors; }
  double Factor(int i) { return this->InteractionFactors[i]; }
  void SetFactor(int i, double x) { this->InteractionFactors[i] = x; }
  // GetLoadBalancing (AbstractQHEOnSphereHamiltonian.cc:3547) caches its segments for a thread count;
  // dropping the cache makes the next product split the architecture's current typical range
  void ResetLoadBalancing()
  {
    delete[] this->LoadBalancingArray;
    this->LoadBalancingArray = 0;
  }
};

// SMPArchitecture whose typical range (AbstractArchitecture.cc:65, [0, dim - 1] in the reference) is a
// window [First, Last] of the space: the rows the reference SMP product splits between its threads
class WindowSMPArchitecture : public SMPArchitecture
{
 public:
  long First, Last;
  WindowSMPArchitecture(int nbrThreads) : SMPArchitecture(nbrThreads), First(0), Last(-1) {}
  void GetTypicalRange(long& minIndex, long& maxIndex)
  {
    if (this->Last >= this->First)
      {
	minIndex = this->First;
	maxIndex = this->Last;
      }
    else
      SMPArchitecture::GetTypicalRange(minIndex, maxIndex);
  }
};

// pseudopotentials: "coulomb" = the reference's LLL Coulomb V_m (EvaluatePseudopotentials,
// PseudoPotentials.cc:35) with the even m set to zero (spin-polarised fermions), else a raw file
static double* PseudopotentialsFromSpec(const char* spec, int lzMax)
{
  if (strcmp(spec, "coulomb") != 0)
    return ReadDoubles(spec, lzMax + 1);
  double* V = EvaluatePseudopotentials(lzMax, 0, 0.0, true);
  for (int m = 0; m <= lzMax; m += 2)
    V[m] = 0.0;
  return V;
}

// J1-J2 periodic chain on a plain Spin1_2Chain (see file header)
class J1J2ChainHarness : public AbstractHamiltonian
{
 protected:
  Spin1_2Chain* Chain;
  int NbrSpin;
  double J1;
  double J2;
  double Shift;
  double* SzSzContributions;

 public:
  J1J2ChainHarness(Spin1_2Chain* chain, int nbrSpin, double j1, double j2)
  {
    this->Chain = chain;
    this->NbrSpin = nbrSpin;
    this->J1 = j1;
    this->J2 = j2;
    this->Shift = 0.0;
    int Dim = this->Chain->GetHilbertSpaceDimension();
    this->SzSzContributions = new double[Dim];
    for (int i = 0; i < Dim; ++i)
      {
	double Tmp = 0.0;
	for (int j = 0; j < this->NbrSpin; ++j)
	  {
	    Tmp += this->J1 * this->Chain->SziSzj(j, (j + 1) % this->NbrSpin, i);
	    Tmp += this->J2 * this->Chain->SziSzj(j, (j + 2) % this->NbrSpin, i);
	  }
	this->SzSzContributions[i] = Tmp;
      }
  }
  ~J1J2ChainHarness() { delete[] this->SzSzContributions; }
  void SetHilbertSpace(AbstractHilbertSpace* hilbertSpace) { this->Chain = (Spin1_2Chain*) hilbertSpace; }
  AbstractHilbertSpace* GetHilbertSpace() { return this->Chain; }
  int GetHilbertSpaceDimension() { return this->Chain->GetHilbertSpaceDimension(); }
  void ShiftHamiltonian(double shift) { this->Shift = shift; }
  bool IsHermitian() { return false; }

  RealVector& LowLevelAddMultiply(RealVector& vSource, RealVector& vDestination, int firstComponent, int nbrComponent)
  {
    int Last = firstComponent + nbrComponent;
    int Dim = this->Chain->GetHilbertSpaceDimension();
    double HalfJ1 = 0.5 * this->J1;
    double HalfJ2 = 0.5 * this->J2;
    double Coef;
    int Pos;
    for (int i = firstComponent; i < Last; ++i)
      {
	double TmpValue = vSource[i];
	vDestination[i] += (this->SzSzContributions[i] + this->Shift) * TmpValue;
	for (int j = 0; j < this->NbrSpin; ++j)
	  {
	    int j1 = (j + 1) % this->NbrSpin;
	    int j2 = (j + 2) % this->NbrSpin;
	    Pos = this->Chain->SmiSpj(j, j1, i, Coef);
	    if (Pos != Dim)
	      vDestination[Pos] += HalfJ1 * Coef * TmpValue;
	    Pos = this->Chain->SmiSpj(j1, j, i, Coef);
	    if (Pos != Dim)
	      vDestination[Pos] += HalfJ1 * Coef * TmpValue;
	    Pos = this->Chain->SmiSpj(j, j2, i, Coef);
	    if (Pos != Dim)
	      vDestination[Pos] += HalfJ2 * Coef * TmpValue;
	    Pos = this->Chain->SmiSpj(j2, j, i, Coef);
	    if (Pos != Dim)
	      vDestination[Pos] += HalfJ2 * Coef * TmpValue;
	  }
      }
    return vDestination;
  }
};

static void WriteEigenvalues(FILE* f, AbstractLanczosAlgorithm* Lanczos, int nev)
{
  RealTriDiagonalSymmetricMatrix TmpMatrix;
  TmpMatrix.Copy(Lanczos->GetDiagonalizedMatrix());
  TmpMatrix.SortMatrixUpOrder();
  for (int i = 0; i < nev; ++i)
    {
      double e = TmpMatrix.DiagonalElement(i);
      fwrite(&e, sizeof(double), 1, f);
    }
}

// the driver loop of QHEOnSphereMainTask.cc:732-753 / GenericRealMainTask.cc:790-808
static void RunLanczosLoop(AbstractHamiltonian* H, AbstractArchitecture* Arch, const char* algo, int nev,
			   int blockSize, int maxIter, double precision, RealVector* initial, int nbrInitial,
			   const char* outName, const char* groundStateName)
{
  AbstractLanczosAlgorithm* Lanczos;
  bool Block = false;
  if (strcmp(algo, "basic") == 0)
    Lanczos = new BasicLanczosAlgorithm(Arch, nev, maxIter);
  else if (strcmp(algo, "full") == 0)
    Lanczos = new FullReorthogonalizedLanczosAlgorithm(Arch, nev, maxIter);
  else if (strcmp(algo, "ground") == 0)
    Lanczos = new BasicLanczosAlgorithmWithGroundState(Arch, maxIter);
  else
    {
      Lanczos = new BasicBlockLanczosAlgorithm(Arch, nev, blockSize, maxIter);
      Block = true;
    }
  if (precision != 0.0)
    Lanczos->SetEigenvaluePrecision(precision);
  Lanczos->SetHamiltonian(H);
  if (Block)
    Lanczos->InitializeLanczosAlgorithm(initial, nbrInitial);
  else
    Lanczos->InitializeLanczosAlgorithm(initial[0]);
  double t0 = Now();
  int CurrentNbrIter;
  Lanczos->RunLanczosAlgorithm(nev + 2);
  if (Block)
    CurrentNbrIter = (nev + 3) * blockSize;
  else
    CurrentNbrIter = nev + 3;
  std::vector<double> History;
  while ((Lanczos->TestConvergence() == false) && (CurrentNbrIter < maxIter))
    {
      if (Block)
	CurrentNbrIter += blockSize;
      else
	++CurrentNbrIter;
      Lanczos->RunLanczosAlgorithm(1);
      RealTriDiagonalSymmetricMatrix TmpMatrix;
      TmpMatrix.Copy(Lanczos->GetDiagonalizedMatrix());
      TmpMatrix.SortMatrixUpOrder();
      History.push_back(TmpMatrix.DiagonalElement(0));
    }
  double t1 = Now();
  int Converged = Lanczos->TestConvergence() ? 1 : 0;
  FILE* f = OpenOut(outName);
  // layout: int32 nev, int32 iterations, int32 converged, double seconds, nev doubles (sorted lowest
  // Ritz values), int32 nbr history, history doubles (lowest Ritz value after each extra step)
  fwrite(&nev, sizeof(int), 1, f);
  fwrite(&CurrentNbrIter, sizeof(int), 1, f);
  fwrite(&Converged, sizeof(int), 1, f);
  double Seconds = t1 - t0;
  fwrite(&Seconds, sizeof(double), 1, f);
  WriteEigenvalues(f, Lanczos, nev);
  int NbrHistory = (int) History.size();
  fwrite(&NbrHistory, sizeof(int), 1, f);
  if (NbrHistory > 0)
    fwrite(&History[0], sizeof(double), NbrHistory, f);
  fclose(f);
  if ((groundStateName != 0) && (strcmp(algo, "ground") == 0))
    {
      RealVector& GS = (RealVector&) Lanczos->GetGroundState();
      GS.WriteVector(groundStateName);
    }
  delete Lanczos;
}

// the driver loop of QHEOnSphereMainTask.cc:671-753 with --disk: BasicLanczosAlgorithmWithDiskStorage
// ("basic") or BasicLanczosAlgorithmWithGroundStateDiskStorage ("ground", ground-state assembly in
// steps of groundIter) run in directory dir, which receives lanczos.dat and the vector files.  start
// = "resume" resumes from dir (ResumeLanczosAlgorithm, no first call, counter from 0), otherwise it
// is the start vector file.  nbrIter bounds the counter as --nbr-iter does in disk mode, so a small
// value leaves an interrupted run on disk.  Output layout as RunLanczosLoop's.
static void RunDiskLanczosLoop(AbstractHamiltonian* H, AbstractArchitecture* Arch, const char* algo, int nbrIter,
			       double precision, const char* dir, const char* start, int groundIter,
			       const char* outName, const char* groundStateName)
{
  AbstractLanczosAlgorithm* Lanczos;
  bool Ground = (strcmp(algo, "ground") == 0);
  // "block<k>": BasicBlockLanczosAlgorithm with --fast-disk (diskFlag), --resume-fastdisk for "resume"
  int BlockSize = (strncmp(algo, "block", 5) == 0) ? atoi(algo + 5) : 0;
  bool Resume = (strcmp(start, "resume") == 0);
  if (Ground)
    Lanczos = new BasicLanczosAlgorithmWithGroundStateDiskStorage(Arch, groundIter, 4000);
  else if (BlockSize > 0)
    Lanczos = new BasicBlockLanczosAlgorithm(Arch, 1, BlockSize, 4000, true, Resume, false, false);
  else
    Lanczos = new BasicLanczosAlgorithmWithDiskStorage(Arch, 1, 4000);
  // start vectors: file names separated by commas (the block gets one per vector)
  std::vector<RealVector> Initial;
  if (!Resume)
    {
      std::string Names(start);
      size_t Pos = 0;
      while (Pos <= Names.size())
	{
	  size_t End = Names.find(',', Pos);
	  if (End == std::string::npos)
	    End = Names.size();
	  RealVector V;
	  V.ReadVector(Names.substr(Pos, End - Pos).c_str());
	  Initial.push_back(V);
	  Pos = End + 1;
	}
    }
  // outputs are opened (or made absolute) before moving into dir
  FILE* f = OpenOut(outName);
  std::string GroundStatePath;
  if (groundStateName != 0)
    {
      GroundStatePath = groundStateName;
      if (groundStateName[0] != '/')
	{
	  char Cwd[4096];
	  if (getcwd(Cwd, sizeof(Cwd)) == 0)
	    exit(2);
	  GroundStatePath = std::string(Cwd) + "/" + groundStateName;
	}
    }
  if (chdir(dir) != 0)
    {
      fprintf(stderr, "cannot enter %s\n", dir);
      exit(2);
    }
  if (precision != 0.0)
    Lanczos->SetEigenvaluePrecision(precision);
  Lanczos->SetHamiltonian(H);
  int CurrentNbrIter = 0;
  double t0 = Now();
  if (BlockSize > 0)
    {
      // QHEOnSphereMainTask.cc:711-736 without --resume: the (resuming) initialisation, then the
      // first call of nbrEigenvalue + 2 block steps
      if (Resume)
	Lanczos->InitializeLanczosAlgorithm();
      else
	Lanczos->InitializeLanczosAlgorithm(&Initial[0], (int) Initial.size());
      Lanczos->RunLanczosAlgorithm(3);
      CurrentNbrIter = 4 * BlockSize;
    }
  else if (Resume)
    Lanczos->ResumeLanczosAlgorithm();
  else
    {
      Lanczos->InitializeLanczosAlgorithm(Initial[0]);
      Lanczos->RunLanczosAlgorithm(3);
      CurrentNbrIter = 4;
    }
  std::vector<double> History;
  while ((Lanczos->TestConvergence() == false) && (CurrentNbrIter < nbrIter))
    {
      CurrentNbrIter += (BlockSize > 0) ? BlockSize : 1;
      Lanczos->RunLanczosAlgorithm(1);
      RealTriDiagonalSymmetricMatrix TmpMatrix;
      TmpMatrix.Copy(Lanczos->GetDiagonalizedMatrix());
      TmpMatrix.SortMatrixUpOrder();
      History.push_back(TmpMatrix.DiagonalElement(0));
    }
  double t1 = Now();
  int Nev = 1;
  int Converged = Lanczos->TestConvergence() ? 1 : 0;
  fwrite(&Nev, sizeof(int), 1, f);
  fwrite(&CurrentNbrIter, sizeof(int), 1, f);
  fwrite(&Converged, sizeof(int), 1, f);
  double Seconds = t1 - t0;
  fwrite(&Seconds, sizeof(double), 1, f);
  WriteEigenvalues(f, Lanczos, Nev);
  int NbrHistory = (int) History.size();
  fwrite(&NbrHistory, sizeof(int), 1, f);
  if (NbrHistory > 0)
    fwrite(&History[0], sizeof(double), NbrHistory, f);
  fclose(f);
  if (Ground && (groundStateName != 0))
    {
      RealVector& GS = (RealVector&) Lanczos->GetGroundState();
      GS.WriteVector(GroundStatePath.c_str());
    }
  delete Lanczos;
}

// REF_THREADS=P (environment) runs the Lanczos commands on SMPArchitecture(P) instead of the
// mono-processor architecture, as the reference programs do with -S --processors P
static AbstractArchitecture* MakeArchitecture()
{
  const char* Env = getenv("REF_THREADS");
  int P = (Env != 0) ? atoi(Env) : 1;
  if (P > 1)
    return new SMPArchitecture(P);
  return new MonoProcessorArchitecture;
}

static void Usage()
{
  fprintf(stderr,
	  "ref_tool commands (all outputs little-endian binary):\n"
	  "  fqhe_basis N 2S 2Lz out\n"
	  "  fqhe_factors N 2S vfile out\n"
	  "  fqhe_rows N 2S 2Lz vfile rowsfile out\n"
	  "  fqhe_matvec N 2S 2Lz vfile xfile shift out\n"
	  "  fqhe_sectors N 2S vfile block maxiter precision fulldiag out\n"
	  "  fqhe_lanczos N 2S 2Lz vfile algo nev block maxiter precision out gsout x0 [x1 ...]\n"
	  "  fqhe_lanczos_disk N 2S 2Lz vfile algo nbriter precision dir x0|resume gsiter out gsout\n"
	  "  fqhe_expect N 2S 2Lz vfile psifile out\n"
	  "  fqhe_entanglement N 2S 2Lz xfile l NA 2LzA out\n"
	  "  fqhe_density N 2S 2Lz xfile l NA 2LzA out\n"
	  "  lfqhe_basis N 2S 2Lz out\n"
	  "  lfqhe_factors N 2S vfile out\n"
	  "  lfqhe_matvec_f N 2S 2Lz vfile ffile xfile shift out\n"
	  "  bqhe_factors N 2S vfile out\n"
	  "  bqhe_matvec_f N 2S 2Lz vfile ffile xfile shift out\n"
	  "  lfqhe_matvec N 2S 2Lz vfile xfile shift out\n"
	  "  lfqhe_lanczos N 2S 2Lz vfile algo nev block maxiter precision out gsout x0 [x1 ...]\n"
	  "  bqhe_basis N 2S 2Lz out\n"
	  "  bqhe_matvec N 2S 2Lz vfile xfile shift out\n"
	  "  bqhe_lanczos N 2S 2Lz vfile algo nev block maxiter precision out gsout x0 [x1 ...]\n"
	  "  fqhe_l2 N 2S 2Lz xfile out\n"
	  "  bqhe_l2 N 2S 2Lz xfile out\n"
	  "  pseudopotentials 2S out\n"
	  "  spin_basis L 2Sz out\n"
	  "  spin_matvec L 2Sz J1 J2 xfile out\n"
	  "  spin_lanczos L 2Sz J1 J2 algo nev block maxiter precision out x0 [x1 ...]\n"
	  "  spint_basis L 2Sz K out\n"
	  "  spint_matvec L 2Sz K J1 J2 xfile out\n"
	  "  spint_lanczos L 2Sz K J1 J2 maxiter precision out x0\n"
	  "  spintc_matvec L 2Sz K J1 J2 xfile out\n"
	  "  spintc_dense L 2Sz K J1 J2 out\n"
	  "  bench_fqhe N 2S 2Lz vspec threads reps hermitian [rows]\n"
	  "  bench_fqhe_block N 2S 2Lz vspec threads reps hermitian k windows\n"
	  "  bench_bqhe N 2S 2Lz vfile threads reps hermitian [rows]\n"
	  "  bench_lfqhe N 2S 2Lz vfile threads reps hermitian [rows]\n"
	  "  bench_spint L 2Sz K J1 J2 threads reps [rows]\n"
	  "  bench_spin L 2Sz J1 J2 threads reps 0\n");
  exit(1);
}

int main(int argc, char** argv)
{
  if (argc < 2)
    Usage();
  const char* Cmd = argv[1];
  cout.precision(17);
  if (strcmp(Cmd, "fqhe_basis") == 0 && argc == 6)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      ExposedFermionOnSphere Space(N, TotalLz, LzMax, 1ul << 20);
      long Dim = Space.GetHilbertSpaceDimension();
      FILE* f = OpenOut(argv[5]);
      fwrite(&Dim, sizeof(long), 1, f);
      for (long i = 0; i < Dim; ++i)
	{
	  unsigned long w = Space.Word(i);
	  fwrite(&w, sizeof(unsigned long), 1, f);
	}
      for (long i = 0; i < Dim; ++i)
	{
	  int l = Space.WordLzMax(i);
	  fwrite(&l, sizeof(int), 1, f);
	}
      // FindStateIndex of every basis word (the TestFindAllStates invariant)
      for (long i = 0; i < Dim; ++i)
	{
	  int idx = Space.Find(Space.Word(i), Space.WordLzMax(i));
	  fwrite(&idx, sizeof(int), 1, f);
	}
      fclose(f);
      return 0;
    }
  // lfqhe_factors: the same tables built on a FermionOnSphereLong space (lzMax up to 126)
  // bqhe_factors: the bosonic tables (BosonOnSphereShort space)
  if ((strcmp(Cmd, "fqhe_factors") == 0 || strcmp(Cmd, "lfqhe_factors") == 0 || strcmp(Cmd, "bqhe_factors") == 0) &&
      argc == 6)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]);
      double* V = ReadDoubles(argv[4], LzMax + 1);
      ParticleOnSphere* SpacePtr;
      if (Cmd[0] == 'l')
	SpacePtr = new FermionOnSphereLong(N, (N & 1) ? 1 : 0, LzMax, 1ul << 20);
      else if (Cmd[0] == 'b')
	SpacePtr = new BosonOnSphereShort(N, ((N * LzMax) & 1) ? 1 : 0, LzMax);
      else
	SpacePtr = new FermionOnSphere(N, (N & 1) ? 1 : 0, LzMax, 1ul << 20);
      MonoProcessorArchitecture Arch;
      ExposedGenericHamiltonian H(SpacePtr, N, LzMax, V, &Arch, false);
      FILE* f = OpenOut(argv[5]);
      // layout: int32 nbrM12, then per pair int32 (m1, m2, nbrM3, m3[nbrM3]); int32 nbrFactors; doubles
      int P = H.GetNbrM12();
      fwrite(&P, sizeof(int), 1, f);
      for (int i = 0; i < P; ++i)
	{
	  int a[3] = {H.M1(i), H.M2(i), H.NbrM3(i)};
	  fwrite(a, sizeof(int), 3, f);
	  for (int j = 0; j < a[2]; ++j)
	    {
	      int m3 = H.M3(i, j);
	      fwrite(&m3, sizeof(int), 1, f);
	    }
	}
      int F = H.NbrFactors();
      fwrite(&F, sizeof(int), 1, f);
      for (int i = 0; i < F; ++i)
	{
	  double x = H.Factor(i);
	  fwrite(&x, sizeof(double), 1, f);
	}
      fclose(f);
      return 0;
    }
  if (strcmp(Cmd, "fqhe_rows") == 0 && argc == 8)
    {
      // the inner loops of AbstractQHEOnSphereHamiltonian::LowLevelAddMultiply (:456-488), one
      // (target, AA sign * AdAd sign, factor index) triple per generated element, in the
      // reference's own enumeration order
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = ReadDoubles(argv[5], LzMax + 1);
      long NbrRows;
      int* Rows = ReadInts(argv[6], NbrRows);
      FermionOnSphere Space(N, TotalLz, LzMax, 1ul << 20);
      MonoProcessorArchitecture Arch;
      ExposedGenericHamiltonian H(&Space, N, LzMax, V, &Arch, false);
      int Dim = Space.GetHilbertSpaceDimension();
      FILE* f = OpenOut(argv[7]);
      // layout: per requested row: int32 row, int32 count, count x (int32 target, int32 sign, int32 factor)
      for (long r = 0; r < NbrRows; ++r)
	{
	  int i = Rows[r];
	  std::vector<int> Out;
	  int FactorIndex = 0;
	  for (int p = 0; p < H.GetNbrM12(); ++p)
	    {
	      double C1 = Space.AA(i, H.M1(p), H.M2(p));
	      if (C1 != 0.0)
		{
		  int Sum = H.M1(p) + H.M2(p);
		  for (int q = 0; q < H.NbrM3(p); ++q)
		    {
		      double C2;
		      int m3 = H.M3(p, q);
		      int Index = Space.AdAd(m3, Sum - m3, C2);
		      if (Index < Dim)
			{
			  Out.push_back(Index);
			  Out.push_back((C1 * C2) > 0.0 ? 1 : -1);
			  Out.push_back(FactorIndex);
			}
		      ++FactorIndex;
		    }
		}
	      else
		FactorIndex += H.NbrM3(p);
	    }
	  int Count = (int) Out.size() / 3;
	  fwrite(&i, sizeof(int), 1, f);
	  fwrite(&Count, sizeof(int), 1, f);
	  if (Count > 0)
	    fwrite(&Out[0], sizeof(int), Out.size(), f);
	}
      fclose(f);
      return 0;
    }
  // FermionOnSphereLong (lzMax up to 126): basis as int64 dimension then (low, high) uint64 per state
  if (strcmp(Cmd, "lfqhe_basis") == 0 && argc == 6)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      ExposedFermionOnSphereLong Space(N, TotalLz, LzMax, 1ul << 20);
      long Dim = Space.GetHilbertSpaceDimension();
      FILE* f = OpenOut(argv[5]);
      fwrite(&Dim, sizeof(long), 1, f);
      for (long i = 0; i < Dim; ++i)
	{
	  unsigned long w[2] = {Space.WordLow(i), Space.WordHigh(i)};
	  fwrite(w, sizeof(unsigned long), 2, f);
	}
      fclose(f);
      return 0;
    }
  if (strcmp(Cmd, "lfqhe_matvec") == 0 && argc == 9)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = ReadDoubles(argv[5], LzMax + 1);
      FermionOnSphereLong Space(N, TotalLz, LzMax, 1ul << 20);
      MonoProcessorArchitecture Arch;
      ParticleOnSphereGenericHamiltonian H(&Space, N, LzMax, V, 0.0, &Arch, 0, false, 0, false);
      H.ShiftHamiltonian(atof(argv[7]));
      RealVector X;
      X.ReadVector(argv[6]);
      RealVector Y(Space.GetHilbertSpaceDimension(), true);
      H.LowLevelMultiply(X, Y);
      Y.WriteVector(argv[8]);
      return 0;
    }
  // the reference's FermionOnSphereLong product with its interaction factors replaced by the ones in
  // ffile (NbrFactors doubles, in the order lfqhe_factors writes them)
  // bqhe_matvec_f: the same for BosonOnSphereShort
  if ((strcmp(Cmd, "lfqhe_matvec_f") == 0 || strcmp(Cmd, "bqhe_matvec_f") == 0) && argc == 10)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = ReadDoubles(argv[5], LzMax + 1);
      ParticleOnSphere* SpacePtr;
      if (Cmd[0] == 'b')
	SpacePtr = new BosonOnSphereShort(N, TotalLz, LzMax);
      else
	SpacePtr = new FermionOnSphereLong(N, TotalLz, LzMax, 1ul << 20);
      ParticleOnSphere& Space = *SpacePtr;
      MonoProcessorArchitecture Arch;
      ExposedGenericHamiltonian H(SpacePtr, N, LzMax, V, &Arch, false);
      double* F = ReadDoubles(argv[6], H.NbrFactors());
      for (int i = 0; i < H.NbrFactors(); ++i)
	H.SetFactor(i, F[i]);
      H.ShiftHamiltonian(atof(argv[8]));
      RealVector X;
      X.ReadVector(argv[7]);
      RealVector Y(Space.GetHilbertSpaceDimension(), true);
      H.LowLevelMultiply(X, Y);
      Y.WriteVector(argv[9]);
      return 0;
    }
  if (strcmp(Cmd, "lfqhe_lanczos") == 0 && argc >= 14)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = ReadDoubles(argv[5], LzMax + 1);
      const char* Algo = argv[6];
      int Nev = atoi(argv[7]), Block = atoi(argv[8]), MaxIter = atoi(argv[9]);
      double Precision = atof(argv[10]);
      FermionOnSphereLong Space(N, TotalLz, LzMax, 9ul << 20);
      AbstractArchitecture* Arch = MakeArchitecture();
      Arch->SetDimension(Space.GetHilbertSpaceDimension());
      ParticleOnSphereGenericHamiltonian H(&Space, N, LzMax, V, 0.0, Arch, 0, false, 0, false);
      int NbrInitial = argc - 13;
      RealVector* Init = new RealVector[NbrInitial];
      for (int i = 0; i < NbrInitial; ++i)
	Init[i].ReadVector(argv[13 + i]);
      RunLanczosLoop(&H, Arch, Algo, Nev, Block, MaxIter, Precision, Init, NbrInitial, argv[11],
		     strcmp(argv[12], "-") == 0 ? 0 : argv[12]);
      return 0;
    }
  if (strcmp(Cmd, "fqhe_matvec") == 0 && argc == 9)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = ReadDoubles(argv[5], LzMax + 1);
      FermionOnSphere Space(N, TotalLz, LzMax, 9ul << 20);
      // REF_THREADS > 1: the SMP product (VectorHamiltonianMultiplyOperation on SMPArchitecture)
      AbstractArchitecture* Arch = MakeArchitecture();
      Arch->SetDimension(Space.GetHilbertSpaceDimension());
      ParticleOnSphereGenericHamiltonian H(&Space, N, LzMax, V, 0.0, Arch, 0, false, 0, false);
      H.ShiftHamiltonian(atof(argv[7]));
      RealVector X;
      X.ReadVector(argv[6]);
      RealVector Y(Space.GetHilbertSpaceDimension(), true);
      VectorHamiltonianMultiplyOperation Op(&H, &X, &Y);
      Op.ApplyOperation(Arch);
      Y.WriteVector(argv[8]);
      return 0;
    }
  if (strcmp(Cmd, "fqhe_sectors") == 0 && argc == 10)
    {
      // every Lz sector 2Lz = Lzmax .. 0 of N fermions (the positive half: 2Lz >= 0), as
      // QHEOnSphereMainTask does per sector: full diagonalisation below `fulldiag` states
      // (GetHamiltonian + Householder + Diagonalize, QHEOnSphereMainTask.cc:397-471), else
      // BasicBlockLanczosAlgorithm with `block` vectors from its own random start
      // (BasicBlockLanczosAlgorithm.cc:233) under the driver loop (QHEOnSphereMainTask.cc:732-753).
      // Output text: per sector "2Lz dim E0 iterations converged method".
      int N = atoi(argv[2]), LzMax = atoi(argv[3]);
      double* V = ReadDoubles(argv[4], LzMax + 1);
      int Block = atoi(argv[5]), MaxIter = atoi(argv[6]);
      double Precision = atof(argv[7]);
      int FullDiag = atoi(argv[8]);
      FILE* f = fopen(argv[9], "w");
      if (f == 0)
	{
	  fprintf(stderr, "cannot open %s\n", argv[9]);
	  exit(2);
	}
      int MaxTwoLz = N * (LzMax - N + 1);
      for (int TwoLz = MaxTwoLz; TwoLz >= 0; TwoLz -= 2)
	{
	  FermionOnSphere Space(N, TwoLz, LzMax, 9ul << 20);
	  long Dim = Space.GetHilbertSpaceDimension();
	  AbstractArchitecture* Arch = MakeArchitecture();
	  Arch->SetDimension(Dim);
	  ParticleOnSphereGenericHamiltonian H(&Space, N, LzMax, V, 0.0, Arch, 0, false, 0, false);
	  double E0;
	  int Iter = 0, Conv = 1;
	  const char* Method;
	  if (Dim < FullDiag)
	    {
	      RealSymmetricMatrix HRep(Dim);
	      H.GetHamiltonian(HRep);
	      if (Dim > 1)
		{
		  RealTriDiagonalSymmetricMatrix TmpTriDiag(Dim);
		  HRep.Householder(TmpTriDiag, 1e-7);
		  TmpTriDiag.Diagonalize();
		  TmpTriDiag.SortMatrixUpOrder();
		  E0 = TmpTriDiag.DiagonalElement(0);
		}
	      else
		HRep.GetMatrixElement(0, 0, E0);
	      Method = "full";
	    }
	  else
	    {
	      BasicBlockLanczosAlgorithm Lanczos(Arch, 1, Block, MaxIter);
	      if (Precision != 0.0)
		Lanczos.SetEigenvaluePrecision(Precision);
	      Lanczos.SetHamiltonian(&H);
	      Lanczos.InitializeLanczosAlgorithm();
	      Lanczos.RunLanczosAlgorithm(3);
	      Iter = 4 * Block;
	      while ((Lanczos.TestConvergence() == false) && (Iter < MaxIter))
		{
		  Iter += Block;
		  Lanczos.RunLanczosAlgorithm(1);
		}
	      Conv = Lanczos.TestConvergence() ? 1 : 0;
	      RealTriDiagonalSymmetricMatrix TmpMatrix;
	      TmpMatrix.Copy(Lanczos.GetDiagonalizedMatrix());
	      TmpMatrix.SortMatrixUpOrder();
	      E0 = TmpMatrix.DiagonalElement(0);
	      Method = "block";
	    }
	  fprintf(f, "%d %ld %.17g %d %d %s\n", TwoLz, Dim, E0, Iter, Conv, Method);
	  fflush(f);
	  delete Arch;
	}
      fclose(f);
      return 0;
    }
  if (strcmp(Cmd, "fqhe_lanczos") == 0 && argc >= 14)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = ReadDoubles(argv[5], LzMax + 1);
      const char* Algo = argv[6];
      int Nev = atoi(argv[7]), Block = atoi(argv[8]), MaxIter = atoi(argv[9]);
      double Precision = atof(argv[10]);
      FermionOnSphere Space(N, TotalLz, LzMax, 9ul << 20);
      AbstractArchitecture* Arch = MakeArchitecture();
      Arch->SetDimension(Space.GetHilbertSpaceDimension());
      ParticleOnSphereGenericHamiltonian H(&Space, N, LzMax, V, 0.0, Arch, 0, false, 0, false);
      int NbrInitial = argc - 13;
      RealVector* Init = new RealVector[NbrInitial];
      for (int i = 0; i < NbrInitial; ++i)
	Init[i].ReadVector(argv[13 + i]);
      RunLanczosLoop(&H, Arch, Algo, Nev, Block, MaxIter, Precision, Init, NbrInitial, argv[11],
		     strcmp(argv[12], "-") == 0 ? 0 : argv[12]);
      return 0;
    }
  // orbital-cut entanglement of a vector (FermionOnSphere.cc:2070, :2474); layout: int64 rows, int64
  // columns, then the matrix row by row (a density matrix is written in full, rows = columns)
  if ((strcmp(Cmd, "fqhe_entanglement") == 0 || strcmp(Cmd, "fqhe_density") == 0) && argc == 10)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      int Cut = atoi(argv[6]), NA = atoi(argv[7]), LzA = atoi(argv[8]);
      FermionOnSphere Space(N, TotalLz, LzMax, 9ul << 20);
      RealVector X;
      X.ReadVector(argv[5]);
      FILE* f = OpenOut(argv[9]);
      if (strcmp(Cmd, "fqhe_entanglement") == 0)
	{
	  RealMatrix M = Space.EvaluatePartialEntanglementMatrix(Cut, NA, LzA, X);
	  long Rows = M.GetNbrRow(), Columns = M.GetNbrColumn();
	  fwrite(&Rows, sizeof(long), 1, f);
	  fwrite(&Columns, sizeof(long), 1, f);
	  for (long i = 0; i < Rows; ++i)
	    for (long j = 0; j < Columns; ++j)
	      {
		double Tmp;
		M.GetMatrixElement(i, j, Tmp);
		fwrite(&Tmp, sizeof(double), 1, f);
	      }
	}
      else
	{
	  RealSymmetricMatrix Rho = Space.EvaluatePartialDensityMatrix(Cut, NA, LzA, X);
	  long Rows = Rho.GetNbrRow();
	  fwrite(&Rows, sizeof(long), 1, f);
	  fwrite(&Rows, sizeof(long), 1, f);
	  for (long i = 0; i < Rows; ++i)
	    for (long j = 0; j < Rows; ++j)
	      {
		double Tmp;
		Rho.GetMatrixElement(i, j, Tmp);
		fwrite(&Tmp, sizeof(double), 1, f);
	      }
	}
      fclose(f);
      return 0;
    }
  // bosons: BosonOnSphereShort with the same Hamiltonian class (its bosonic factors and AA / AdAd)
  if (strcmp(Cmd, "bqhe_basis") == 0 && argc == 6)
    {
      // layout: int64 dimension, then per state the occupations n_0..n_2S as int32 (PrintState)
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      BosonOnSphereShort Space(N, TotalLz, LzMax);
      long Dim = Space.GetHilbertSpaceDimension();
      FILE* f = OpenOut(argv[5]);
      fwrite(&Dim, sizeof(long), 1, f);
      for (long i = 0; i < Dim; ++i)
	{
	  std::ostringstream Str;
	  Space.PrintState(Str, (int) i);
	  std::istringstream In(Str.str());
	  for (int m = 0; m <= LzMax; ++m)
	    {
	      int Occupation = -1;
	      In >> Occupation;
	      fwrite(&Occupation, sizeof(int), 1, f);
	    }
	}
      fclose(f);
      return 0;
    }
  if (strcmp(Cmd, "bqhe_matvec") == 0 && argc == 9)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = ReadDoubles(argv[5], LzMax + 1);
      BosonOnSphereShort Space(N, TotalLz, LzMax);
      MonoProcessorArchitecture Arch;
      ParticleOnSphereGenericHamiltonian H(&Space, N, LzMax, V, 0.0, &Arch, 0, false, 0, false);
      H.ShiftHamiltonian(atof(argv[7]));
      RealVector X;
      X.ReadVector(argv[6]);
      RealVector Y(Space.GetHilbertSpaceDimension(), true);
      H.LowLevelMultiply(X, Y);
      Y.WriteVector(argv[8]);
      return 0;
    }
  if (strcmp(Cmd, "bqhe_lanczos") == 0 && argc >= 14)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = ReadDoubles(argv[5], LzMax + 1);
      int Nev = atoi(argv[7]), Block = atoi(argv[8]), MaxIter = atoi(argv[9]);
      BosonOnSphereShort Space(N, TotalLz, LzMax);
      AbstractArchitecture* Arch = MakeArchitecture();
      Arch->SetDimension(Space.GetHilbertSpaceDimension());
      ParticleOnSphereGenericHamiltonian H(&Space, N, LzMax, V, 0.0, Arch, 0, false, 0, false);
      int NbrInitial = argc - 13;
      RealVector* Init = new RealVector[NbrInitial];
      for (int i = 0; i < NbrInitial; ++i)
	Init[i].ReadVector(argv[13 + i]);
      RunLanczosLoop(&H, Arch, argv[6], Nev, Block, MaxIter, atof(argv[10]), Init, NbrInitial, argv[11],
		     strcmp(argv[12], "-") == 0 ? 0 : argv[12]);
      return 0;
    }
  if (strcmp(Cmd, "fqhe_lanczos_disk") == 0 && argc == 14)
    {
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = ReadDoubles(argv[5], LzMax + 1);
      FermionOnSphere Space(N, TotalLz, LzMax, 9ul << 20);
      AbstractArchitecture* Arch = MakeArchitecture();
      Arch->SetDimension(Space.GetHilbertSpaceDimension());
      ParticleOnSphereGenericHamiltonian H(&Space, N, LzMax, V, 0.0, Arch, 0, false, 0, false);
      RunDiskLanczosLoop(&H, Arch, argv[6], atoi(argv[7]), atof(argv[8]), argv[9], argv[10], atoi(argv[11]),
			 argv[12], strcmp(argv[13], "-") == 0 ? 0 : argv[13]);
      return 0;
    }
  if (strcmp(Cmd, "fqhe_expect") == 0 && argc == 8)
    {
      // <psi|H_m|psi> for every m, with H_m the generic Hamiltonian of V = e_m (linearity of
      // EvaluateInteractionFactors in V), followed by <psi|H(V)|psi> for the given V
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = ReadDoubles(argv[5], LzMax + 1);
      FermionOnSphere Space(N, TotalLz, LzMax, 1ul << 20);
      MonoProcessorArchitecture Arch;
      RealVector Psi;
      Psi.ReadVector(argv[6]);
      RealVector Tmp(Space.GetHilbertSpaceDimension(), true);
      FILE* f = OpenOut(argv[7]);
      double* E = new double[LzMax + 1];
      for (int m = 0; m <= LzMax; ++m)
	{
	  for (int k = 0; k <= LzMax; ++k)
	    E[k] = (k == m) ? 1.0 : 0.0;
	  ParticleOnSphereGenericHamiltonian Hm(&Space, N, LzMax, E, 0.0, &Arch, 0, false, 0, false);
	  Hm.LowLevelMultiply(Psi, Tmp);
	  double x = (Psi * Tmp) / (Psi * Psi);
	  fwrite(&x, sizeof(double), 1, f);
	}
      ParticleOnSphereGenericHamiltonian H(&Space, N, LzMax, V, 0.0, &Arch, 0, false, 0, false);
      H.LowLevelMultiply(Psi, Tmp);
      double x = (Psi * Tmp) / (Psi * Psi);
      fwrite(&x, sizeof(double), 1, f);
      fclose(f);
      return 0;
    }
  if (strcmp(Cmd, "fqhe_l2") == 0 && argc == 7)
    {
      // y = L^2 x with the reference's ParticleOnSphereL2Hamiltonian (l2Factor 1, Lz fixed by the
      // sector, on the fly, hermitian symmetry off)
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      FermionOnSphere Space(N, TotalLz, LzMax, 1ul << 20);
      MonoProcessorArchitecture Arch;
      RealVector X;
      X.ReadVector(argv[5]);
      RealVector Y(Space.GetHilbertSpaceDimension(), true);
      ParticleOnSphereL2Hamiltonian L2(&Space, N, LzMax, TotalLz, &Arch, 1.0, 0, true, false, 0, false);
      L2.LowLevelMultiply(X, Y);
      Y.WriteVector(argv[6]);
      return 0;
    }
  if (strcmp(Cmd, "bqhe_l2") == 0 && argc == 7)
    {
      // the same L^2 product on a BosonOnSphereShort space (the operator's bosonic branch)
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      BosonOnSphereShort Space(N, TotalLz, LzMax);
      MonoProcessorArchitecture Arch;
      RealVector X;
      X.ReadVector(argv[5]);
      RealVector Y(Space.GetHilbertSpaceDimension(), true);
      ParticleOnSphereL2Hamiltonian L2(&Space, N, LzMax, TotalLz, &Arch, 1.0, 0, true, false, 0, false);
      L2.LowLevelMultiply(X, Y);
      Y.WriteVector(argv[6]);
      return 0;
    }
  if (strcmp(Cmd, "pseudopotentials") == 0 && argc == 4)
    {
      int NbrFlux = atoi(argv[2]);
      double* V = EvaluatePseudopotentials(NbrFlux, 0, 0.0, true);
      FILE* f = OpenOut(argv[3]);
      fwrite(V, sizeof(double), NbrFlux + 1, f);
      fclose(f);
      return 0;
    }
  if (strcmp(Cmd, "spin_basis") == 0 && argc == 5)
    {
      int L = atoi(argv[2]), Sz = atoi(argv[3]);
      ExposedSpin1_2Chain Chain(L, Sz, 1 << 20);
      long Dim = Chain.GetHilbertSpaceDimension();
      FILE* f = OpenOut(argv[4]);
      fwrite(&Dim, sizeof(long), 1, f);
      for (long i = 0; i < Dim; ++i)
	{
	  unsigned long w = Chain.Word(i);
	  fwrite(&w, sizeof(unsigned long), 1, f);
	}
      for (long i = 0; i < Dim; ++i)
	{
	  int idx = Chain.Find(Chain.Word(i));
	  fwrite(&idx, sizeof(int), 1, f);
	}
      fclose(f);
      return 0;
    }
  if (strcmp(Cmd, "spin_matvec") == 0 && argc == 8)
    {
      int L = atoi(argv[2]), Sz = atoi(argv[3]);
      Spin1_2Chain Chain(L, Sz, 1 << 20);
      J1J2ChainHarness H(&Chain, L, atof(argv[4]), atof(argv[5]));
      RealVector X;
      X.ReadVector(argv[6]);
      RealVector Y(Chain.GetHilbertSpaceDimension(), true);
      H.LowLevelMultiply(X, Y);
      Y.WriteVector(argv[7]);
      return 0;
    }
  // translations: Spin1_2ChainWithTranslations(L, K, 1, 2Sz) with SpinChainJ1J2RealHamiltonianWithTranslations
  // (real: K = 0 or L / 2)
  if (strcmp(Cmd, "spint_basis") == 0 && argc == 6)
    {
      // layout: int64 dimension, then the states (PrintState's hexadecimal word) as uint64
      int L = atoi(argv[2]), Sz = atoi(argv[3]), K = atoi(argv[4]);
      Spin1_2ChainWithTranslations Chain(L, K, 1, Sz, 1 << 20, 1 << 20);
      long Dim = Chain.GetHilbertSpaceDimension();
      FILE* f = OpenOut(argv[5]);
      fwrite(&Dim, sizeof(long), 1, f);
      for (long i = 0; i < Dim; ++i)
	{
	  std::ostringstream Str;
	  Chain.PrintState(Str, (int) i);
	  std::string Text = Str.str();
	  unsigned long Word = strtoul(Text.substr(Text.rfind(' ') + 1).c_str(), 0, 16);
	  fwrite(&Word, sizeof(unsigned long), 1, f);
	}
      fclose(f);
      return 0;
    }
  if (strcmp(Cmd, "spint_matvec") == 0 && argc == 9)
    {
      int L = atoi(argv[2]), Sz = atoi(argv[3]), K = atoi(argv[4]);
      Spin1_2ChainWithTranslations Chain(L, K, 1, Sz, 1 << 20, 1 << 20);
      SpinChainJ1J2RealHamiltonianWithTranslations H(&Chain, L, atof(argv[5]), atof(argv[6]));
      RealVector X;
      X.ReadVector(argv[7]);
      RealVector Y(Chain.GetHilbertSpaceDimension(), true);
      H.LowLevelMultiply(X, Y);
      Y.WriteVector(argv[8]);
      return 0;
    }
  // complex momentum sectors: SpinChainJ1J2HamiltonianWithTranslations on ComplexVector (any K)
  if (strcmp(Cmd, "spintc_matvec") == 0 && argc == 9)
    {
      int L = atoi(argv[2]), Sz = atoi(argv[3]), K = atoi(argv[4]);
      Spin1_2ChainWithTranslations Chain(L, K, 1, Sz, 1 << 20, 1 << 20);
      SpinChainJ1J2HamiltonianWithTranslations H(&Chain, L, atof(argv[5]), atof(argv[6]));
      ComplexVector X;
      X.ReadVector(argv[7]);
      ComplexVector Y(Chain.GetHilbertSpaceDimension(), true);
      H.LowLevelMultiply(X, Y);
      Y.WriteVector(argv[8]);
      return 0;
    }
  // the dense matrix of that product, column by column (int64 dim, then dim x dim complex, row-major)
  if (strcmp(Cmd, "spintc_dense") == 0 && argc == 8)
    {
      int L = atoi(argv[2]), Sz = atoi(argv[3]), K = atoi(argv[4]);
      Spin1_2ChainWithTranslations Chain(L, K, 1, Sz, 1 << 20, 1 << 20);
      SpinChainJ1J2HamiltonianWithTranslations H(&Chain, L, atof(argv[5]), atof(argv[6]));
      long Dim = Chain.GetHilbertSpaceDimension();
      std::vector<double> M(2 * Dim * Dim, 0.0);
      ComplexVector X(Dim, true), Y(Dim, true);
      for (long c = 0; c < Dim; ++c)
	{
	  X.ClearVector();
	  X[c] = Complex(1.0, 0.0);
	  H.LowLevelMultiply(X, Y);
	  for (long r = 0; r < Dim; ++r)
	    {
	      M[2 * (r * Dim + c)] = Y[r].Re;
	      M[2 * (r * Dim + c) + 1] = Y[r].Im;
	    }
	}
      FILE* f = OpenOut(argv[7]);
      fwrite(&Dim, sizeof(long), 1, f);
      fwrite(M.data(), sizeof(double), M.size(), f);
      fclose(f);
      return 0;
    }
  if (strcmp(Cmd, "spint_lanczos") == 0 && argc == 11)
    {
      int L = atoi(argv[2]), Sz = atoi(argv[3]), K = atoi(argv[4]);
      Spin1_2ChainWithTranslations Chain(L, K, 1, Sz, 1 << 20, 1 << 20);
      SpinChainJ1J2RealHamiltonianWithTranslations H(&Chain, L, atof(argv[5]), atof(argv[6]));
      AbstractArchitecture* Arch = MakeArchitecture();
      Arch->SetDimension(Chain.GetHilbertSpaceDimension());
      RealVector* Init = new RealVector[1];
      Init[0].ReadVector(argv[10]);
      RunLanczosLoop(&H, Arch, "basic", 1, 1, atoi(argv[7]), atof(argv[8]), Init, 1, argv[9], 0);
      return 0;
    }
  if (strcmp(Cmd, "spin_lanczos") == 0 && argc >= 13)
    {
      int L = atoi(argv[2]), Sz = atoi(argv[3]);
      Spin1_2Chain Chain(L, Sz, 1 << 20);
      J1J2ChainHarness H(&Chain, L, atof(argv[4]), atof(argv[5]));
      AbstractArchitecture* Arch = MakeArchitecture();
      Arch->SetDimension(Chain.GetHilbertSpaceDimension());
      const char* Algo = argv[6];
      int Nev = atoi(argv[7]), Block = atoi(argv[8]), MaxIter = atoi(argv[9]);
      double Precision = atof(argv[10]);
      int NbrInitial = argc - 12;
      RealVector* Init = new RealVector[NbrInitial];
      for (int i = 0; i < NbrInitial; ++i)
	Init[i].ReadVector(argv[12 + i]);
      RunLanczosLoop(&H, Arch, Algo, Nev, Block, MaxIter, Precision, Init, NbrInitial, argv[11], 0);
      return 0;
    }
  if ((strcmp(Cmd, "bench_fqhe") == 0 || strcmp(Cmd, "bench_bqhe") == 0 || strcmp(Cmd, "bench_lfqhe") == 0) &&
      (argc == 9 || argc == 10))
    {
      // bench_bqhe: the same with BosonOnSphereShort; bench_lfqhe: with FermionOnSphereLong
      // times the reference SMP matvec: VectorHamiltonianMultiplyOperation on SMPArchitecture
      // (VectorHamiltonianMultiplyOperation.cc:241-320), on-the-fly (memory 0) as with -m 0.
      // An optional row count bounds the sample: the architecture's typical range (the rows the
      // SMP operation splits between its threads, AbstractArchitecture.cc:65) is set to the first
      // `rows` rows instead of the whole space.
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = PseudopotentialsFromSpec(argv[5], LzMax);
      int Threads = atoi(argv[6]);
      int Reps = atoi(argv[7]);
      bool Hermitian = atoi(argv[8]) != 0;
      double ts = Now();
      ParticleOnSphere* SpacePtr;
      if (strcmp(Cmd, "bench_bqhe") == 0)
	SpacePtr = new BosonOnSphereShort(N, TotalLz, LzMax);
      else if (strcmp(Cmd, "bench_lfqhe") == 0)
	SpacePtr = new FermionOnSphereLong(N, TotalLz, LzMax, 9ul << 20);
      else
	SpacePtr = new FermionOnSphere(N, TotalLz, LzMax, 9ul << 20);
      ParticleOnSphere& Space = *SpacePtr;
      SMPArchitecture Arch(Threads);
      long Dim = Space.GetHilbertSpaceDimension();
      long Rows = (argc == 10) ? atol(argv[9]) : Dim;
      if (Rows <= 0 || Rows > Dim)
	Rows = Dim;
      Arch.SetDimension(Rows);
      ParticleOnSphereGenericHamiltonian H(SpacePtr, N, LzMax, V, 0.0, &Arch, 0, false, 0, Hermitian);
      double tsetup = Now() - ts;
      RealVector X(Dim, true), Y(Dim, true);
      for (long i = 0; i < Dim; ++i)
	X[i] = 1.0 / sqrt((double) Dim);
      double Best = 1e30, Total = 0.0, Check = 0.0;
      for (int r = 0; r < Reps; ++r)
	{
	  VectorHamiltonianMultiplyOperation Op(&H, &X, &Y);
	  double t0 = Now();
	  Op.ApplyOperation(&Arch);
	  double t = Now() - t0;
	  Total += t;
	  if (t < Best)
	    Best = t;
	  Check = X * Y;
	}
      printf("{\"dim\": %ld, \"rows\": %ld, \"threads\": %d, \"reps\": %d, \"best_s\": %.6e, \"mean_s\": %.6e, "
	     "\"setup_s\": %.3f, \"hermitian\": %d, \"xHx\": %.15e}\n", Dim, Rows, Threads, Reps, Best, Total / Reps,
	     tsetup, Hermitian ? 1 : 0, Check);
      return 0;
    }
  if (strcmp(Cmd, "bench_fqhe_block") == 0 && argc == 11)
    {
      // times the reference SMP block product of block Lanczos: MultipleVectorHamiltonianMultiplyOperation
      // (MultipleVectorHamiltonianMultiplyOperation.cc:56, SMP split :555-640) on k vectors, on the fly
      // (memory 0, as with -m 0), hermitian as the Hamiltonian says (:73-79) ->
      // HermitianLowLevelMultipleMultiply (AbstractQHEOnSphereHamiltonian.cc:3019).  The space is cut
      // into `windows` equal row windows; repetition r multiplies window r mod windows (all windows
      // together are one whole product).  vspec: "coulomb" or a raw file of 2S + 1 doubles.
      int N = atoi(argv[2]), LzMax = atoi(argv[3]), TotalLz = atoi(argv[4]);
      double* V = PseudopotentialsFromSpec(argv[5], LzMax);
      int Threads = atoi(argv[6]);
      int Reps = atoi(argv[7]);
      bool Hermitian = atoi(argv[8]) != 0;
      int K = atoi(argv[9]);
      long Windows = atol(argv[10]);
      double ts = Now();
      FermionOnSphere Space(N, TotalLz, LzMax, 9ul << 20);
      WindowSMPArchitecture Arch(Threads);
      long Dim = Space.GetHilbertSpaceDimension();
      if (Windows < 1 || Windows > Dim)
	Windows = 1;
      Arch.SetDimension(Dim);
      ExposedGenericHamiltonian H(&Space, N, LzMax, V, &Arch, Hermitian);
      double tsetup = Now() - ts;
      RealVector* X = new RealVector[K];
      RealVector* Y = new RealVector[K];
      for (int j = 0; j < K; ++j)
	{
	  X[j] = RealVector(Dim, true);
	  Y[j] = RealVector(Dim, true);
	  for (long i = 0; i < Dim; ++i)
	    X[j][i] = (1.0 + 0.25 * j * ((i % 7) - 3.0)) / sqrt((double) Dim);
	}
      printf("{\"dim\": %ld, \"threads\": %d, \"k\": %d, \"windows\": %ld, \"hermitian\": %d, \"setup_s\": %.3f, "
	     "\"reps\": [", Dim, Threads, K, Windows, Hermitian ? 1 : 0, tsetup);
      for (int r = 0; r < Reps; ++r)
	{
	  long w = r % Windows;
	  Arch.First = (Dim * w) / Windows;
	  Arch.Last = (Dim * (w + 1)) / Windows - 1;
	  H.ResetLoadBalancing();
	  MultipleVectorHamiltonianMultiplyOperation Op(&H, X, Y, K);
	  double t0 = Now();
	  Op.ApplyOperation(&Arch);
	  double t = Now() - t0;
	  double Check = 0.0;
	  for (int j = 0; j < K; ++j)
	    Check += X[j] * Y[j];
	  printf("%s{\"first\": %ld, \"rows\": %ld, \"s\": %.6e, \"xHx\": %.15e}", r ? ", " : "", Arch.First,
		 Arch.Last - Arch.First + 1, t, Check);
	  fflush(stdout);
	}
      printf("]}\n");
      return 0;
    }
  if (strcmp(Cmd, "bench_spint") == 0 && (argc == 9 || argc == 10))
    {
      // the reference SMP product of SpinChainJ1J2RealHamiltonianWithTranslations on a momentum sector,
      // over the first `rows` rows when given (as bench_bqhe)
      int L = atoi(argv[2]), Sz = atoi(argv[3]), K = atoi(argv[4]);
      int Threads = atoi(argv[7]);
      int Reps = atoi(argv[8]);
      double ts = Now();
      Spin1_2ChainWithTranslations Chain(L, K, 1, Sz, 1 << 20, 1 << 20);
      SMPArchitecture Arch(Threads);
      long Dim = Chain.GetHilbertSpaceDimension();
      long Rows = (argc == 10) ? atol(argv[9]) : Dim;
      if (Rows <= 0 || Rows > Dim)
	Rows = Dim;
      Arch.SetDimension(Rows);
      SpinChainJ1J2RealHamiltonianWithTranslations H(&Chain, L, atof(argv[5]), atof(argv[6]));
      double tsetup = Now() - ts;
      RealVector X(Dim, true), Y(Dim, true);
      for (long i = 0; i < Dim; ++i)
	X[i] = 1.0 / sqrt((double) Dim);
      double Best = 1e30, Total = 0.0, Check = 0.0;
      for (int r = 0; r < Reps; ++r)
	{
	  VectorHamiltonianMultiplyOperation Op(&H, &X, &Y);
	  double t0 = Now();
	  Op.ApplyOperation(&Arch);
	  double t = Now() - t0;
	  Total += t;
	  if (t < Best)
	    Best = t;
	  Check = X * Y;
	}
      printf("{\"dim\": %ld, \"rows\": %ld, \"threads\": %d, \"reps\": %d, \"best_s\": %.6e, \"mean_s\": %.6e, "
	     "\"setup_s\": %.3f, \"xHx\": %.15e}\n", Dim, Rows, Threads, Reps, Best, Total / Reps, tsetup, Check);
      return 0;
    }
  if (strcmp(Cmd, "bench_spin") == 0 && argc == 9)
    {
      int L = atoi(argv[2]), Sz = atoi(argv[3]);
      int Threads = atoi(argv[6]);
      int Reps = atoi(argv[7]);
      (void) argv[8];
      double ts = Now();
      Spin1_2Chain Chain(L, Sz, 1 << 26);
      J1J2ChainHarness H(&Chain, L, atof(argv[4]), atof(argv[5]));
      SMPArchitecture Arch(Threads);
      Arch.SetDimension(Chain.GetHilbertSpaceDimension());
      double tsetup = Now() - ts;
      long Dim = Chain.GetHilbertSpaceDimension();
      RealVector X(Dim, true), Y(Dim, true);
      for (long i = 0; i < Dim; ++i)
	X[i] = 1.0 / sqrt((double) Dim);
      double Best = 1e30, Total = 0.0, Check = 0.0;
      for (int r = 0; r < Reps; ++r)
	{
	  VectorHamiltonianMultiplyOperation Op(&H, &X, &Y);
	  double t0 = Now();
	  Op.ApplyOperation(&Arch);
	  double t = Now() - t0;
	  Total += t;
	  if (t < Best)
	    Best = t;
	  Check = X * Y;
	}
      printf("{\"dim\": %ld, \"threads\": %d, \"reps\": %d, \"best_s\": %.6e, \"mean_s\": %.6e, "
	     "\"setup_s\": %.3f, \"xHx\": %.15e}\n", Dim, Threads, Reps, Best, Total / Reps, tsetup, Check);
      return 0;
    }
  Usage();
  return 1;
}
