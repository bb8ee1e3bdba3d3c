// Chemistry kernels (k_chem_cells, k_chem_batch) in their own translation unit.
#include <stdexcept>
#include "ocfd_chem.cuh"
#include "ocfd_launch.h"

namespace ocfd {
int current_const_p();  // the batched reactors' form (ocfd_gpu.cu): 1 constant pressure, 0 constant volume
int current_timeadv();  // CHEM_TimeAdv of the current set-up
int current_mech();     // the mechanism form of the chemistry kernels (MECH_GENERIC or a compiled one)

int mech_match(const DevConst& c) {
  namespace m = mech_h2air9;
  if (c.ns != m::NS || c.nreac != m::NR || c.rereac != m::REREAC) return MECH_GENERIC;
  for (int j = 0; j < m::NR; j++) {
    if (c.af_type[j] != m::AF_TYPE[j] || c.tr_reac[j] != m::TR_REAC[j]) return MECH_GENERIC;
    int sg = 0;
    for (int i = 0; i < m::NS; i++) {
      if (c.vf[j][i] != m::VF[j][i] || c.vr[j][i] != m::VR[j][i]) return MECH_GENERIC;
      sg += m::VR[j][i] - m::VF[j][i];
    }
    if (c.sgm[j] != sg) return MECH_GENERIC;
  }
  return MECH_H2AIR9;
}

#define NS_CASES(...)                                          \
  switch (ns) {                                                \
    case 1: { constexpr int NSV = 1; __VA_ARGS__; } break;     \
    case 2: { constexpr int NSV = 2; __VA_ARGS__; } break;     \
    case 3: { constexpr int NSV = 3; __VA_ARGS__; } break;     \
    case 4: { constexpr int NSV = 4; __VA_ARGS__; } break;     \
    case 5: { constexpr int NSV = 5; __VA_ARGS__; } break;     \
    case 6: { constexpr int NSV = 6; __VA_ARGS__; } break;     \
    case 7: { constexpr int NSV = 7; __VA_ARGS__; } break;     \
    case 8: { constexpr int NSV = 8; __VA_ARGS__; } break;     \
    case 9: { constexpr int NSV = 9; __VA_ARGS__; } break;     \
    default: throw std::runtime_error("N_SPEC must be 1..9");  \
  }

void launch_chem_cells(int ns, long long ncell, double* f, double* Et, double* T, double* p, double* di, double dt2,
                       int nsub, int* nfail, cudaStream_t st) {
  unsigned nb = (unsigned)((ncell + OCFD_CHEM_TPB - 1) / OCFD_CHEM_TPB);
  if (ns == mech_h2air9::NS && current_timeadv() == -1 && current_mech() == MECH_H2AIR9) {
    k_chem_cells<mech_h2air9::NS, MECH_H2AIR9><<<nb, OCFD_CHEM_TPB, 0, st>>>(f, Et, T, p, di, dt2, nsub, nfail);
    return;
  }
  NS_CASES(k_chem_cells<NSV><<<nb, OCFD_CHEM_TPB, 0, st>>>(f, Et, T, p, di, dt2, nsub, nfail));
}

void launch_chem_batch(int ns, int sms, int n, double* di, double* e, const double* dt, const int* nsub,
                       const int* perm, int* counter, int* nfail, cudaStream_t st) {
  const bool cp = current_const_p() != 0;
  // A batch that cannot fill the GPU with one reactor per thread (fewer reactors than the serial
  // kernel's resident threads, e.g. the reactors the surrogate's gate rejects) is latency bound:
  // its time is that of its stiffest reactor's sub-steps on one thread. It runs the linearised
  // implicit Euler on the warp-cooperative kernel instead (the same numbers bit for bit, a group of
  // lanes per reactor: a fraction of the latency per sub-step). Large batches keep the serial
  // kernel, which has 5x its throughput (measured on 2^20 reactors: 58 against 325 ms).
  int cap = 0;
  NS_CASES({
    int per = 0;
    if (cp) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_chem_batch<NSV, true>, OCFD_CHEM_TPB, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_chem_batch<NSV, false>, OCFD_CHEM_TPB, 0);
    cap = sms * (per < 1 ? 1 : per) * OCFD_CHEM_TPB;
  });
  if (current_timeadv() == -1 && ns >= 2 && n < cap) {
    NS_CASES({
      if constexpr (NSV >= 2) {
        int per = 0;
        if (cp) {
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_chem_batch_coop<NSV, true>, COOP_THREADS, 0);
          if (per < 1) per = 1;
          k_chem_batch_coop<NSV, true><<<sms * per, COOP_THREADS, 0, st>>>(n, di, e, dt, nsub, perm, counter, nfail);
        } else {
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_chem_batch_coop<NSV, false>, COOP_THREADS, 0);
          if (per < 1) per = 1;
          k_chem_batch_coop<NSV, false><<<sms * per, COOP_THREADS, 0, st>>>(n, di, e, dt, nsub, perm, counter, nfail);
        }
      }
    });
    return;
  }
  auto serial = [&](auto kern) {
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, OCFD_CHEM_TPB, 0);
    if (per < 1) per = 1;
    kern<<<sms * per, OCFD_CHEM_TPB, 0, st>>>(n, di, e, dt, nsub, perm, counter, nfail);
  };
  if (ns == mech_h2air9::NS && current_timeadv() == -1 && current_mech() == MECH_H2AIR9) {
    constexpr int M = mech_h2air9::NS;
    if (cp) serial(k_chem_batch<M, true, MECH_H2AIR9>);
    else serial(k_chem_batch<M, false, MECH_H2AIR9>);
    return;
  }
  NS_CASES({
    if (cp) serial(k_chem_batch<NSV, true>);
    else serial(k_chem_batch<NSV, false>);
  });
}
}  // namespace ocfd
