// Files in the reference's formats: vector files and the lanczos.dat state files of the
// disk-storage Lanczos classes (host code, disk_formats.cc).
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

namespace dh {

std::string join_path(const std::string& directory, const char* name);

// RealVector::WriteVector / ReadVector (src/Vector/RealVector.cc:3669, :3798), host arrays
int vector_file_write(const std::string& path, const double* v, int64_t dim, int per = 1);
int vector_file_read(const std::string& path, double* v, int64_t dim, int per = 1);
int vector_file_dimension(const std::string& path, int64_t* dim, int per = 1);

// The fields of lanczos.dat.  algorithm DH_LANCZOS_BASIC: BasicLanczosAlgorithmWithDiskStorage
// (Index, PreviousLastWantedEigenvalue, EigenvaluePrecision, NbrRow, the three vector file names,
// diagonal 0..Index+1, upper diagonal 0..Index); DH_LANCZOS_WITH_GROUND_STATE:
// BasicLanczosAlgorithmWithGroundStateDiskStorage (Index, GroundStateEvaluationFlag,
// PreviousLastWantedEigenvalue, EigenvaluePrecision, NbrEigenvalue, NbrRow, NbrRow diagonal and
// NbrRow - 1 upper-diagonal elements).
struct LanczosDiskState {
  int index = 0;
  int ground_flag = 0;
  double prev_last = 0.0;
  double precision = 0.0;
  int nbr_eigenvalue = 1;
  int nbr_row = 0;
  char names[3][8] = {{0}, {0}, {0}};
  std::vector<double> diag, upper;
};
int lanczos_state_write(const std::string& path, int algorithm, const LanczosDiskState& s);
int lanczos_state_read(const std::string& path, int algorithm, LanczosDiskState* s);

}  // namespace dh
