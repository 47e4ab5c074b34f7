// remdgpu.h -- drop-in replacement for the reference's src/remdgpu.h.
//
// Same class name and public members as REMDGPU (src/remdgpu.h:92-238), so the
// reference's REMD driver (src/remd.cxx:114-119, 241-269, 309, 414, 425, 444)
// compiles unchanged with -DENABLE_GPU; every member forwards to the C-ABI of
// libremd_b200.so (include/remd_b200.h).  Unlike the reference, no vgg_common.h
// is needed and CUDA errors are reported instead of ignored: a failing call
// prints remd_last_error() and exits, which is what the reference's driver
// expects of a fatal GPU error (src/remdgpu.cu:208-212).
#ifndef H_REMDGPU
#define H_REMDGPU

#include <cassert>
#include <ostream>
#include <vector>

#include "molecules.h"
#include "integrator.h"
#include "remdinfo.h"
#include "remd_b200.h"

class REMDGPU {
 public:
  REMDGPU(Molecules** mlcls, const unsigned int nreplica);
  ~REMDGPU();
  void ExecuteSteps(double* T, double* P);
  void GetBackAllVariablesFromGPU();
  void OutputCheckPoint(const char* prefix, const int* index);
  void OutputCDV(const char* prefix, const unsigned int step, const int* index);
  void ConvertVariablesToHost(Molecules** mlcls);
  float GetPotential(unsigned int rep);
  float GetVolume(unsigned int rep);
  Average GetAverages(unsigned int rep);
  void PrintAll(std::ostream& os);
  void Diff(Molecules** mlcls, std::ostream& os);

 private:
  remd_handle h_ = nullptr;
  unsigned int nreplica_ = 0;
  int nmol_ = 0;
  std::vector<double> avg_;
  void check(remd_status st, const char* what);
};

#endif
