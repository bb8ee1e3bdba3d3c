// NS_solver of the reference (code/flow-solver/OCFD_NS_Solver.f90:9-70) as a compiled host program
// over the library's C ABI: the same call sequence a Fortran driver patched with the iso_c_binding
// module makes. It reads a case file written by ocfd_b200.cases.Case.save (the parameter records,
// grid, initial primitives and boundary tables of one run), advances nsteps Strang steps
//   flow_time_advance(dt/2)  ->  Chemical_time_advance(dt/nsub) x nsub + comput_T_P  ->  flow_time_advance(dt/2)
// after every step calls filtering (:48) and OCFD_analysis (:55; ana_box rows appended to
// statistics.dat, Q-<Istep>.dat, time averages and their OCFD-comb<Istep>.dat.average files, in
// the working directory as the reference writes them), prints show_flow_msg every Istep_show
// steps, and writes the final f, di and primitives.
//
//   ocfd_ns_solver <case file> <output file>
//   ocfd_ns_solver --describe <case file>     (reads the case and prints its sizes; no device work)
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ocfd_gpu.h"

namespace {

struct Reader {
  FILE* f;
  explicit Reader(const char* path) : f(std::fopen(path, "rb")) {}
  ~Reader() {
    if (f) std::fclose(f);
  }
  template <class T>
  T get() {
    T v{};
    if (std::fread(&v, sizeof(T), 1, f) != 1) throw std::string("case file truncated");
    return v;
  }
  void bytes(void* dst, size_t n) {
    if (n && std::fread(dst, 1, n, f) != n) throw std::string("case file truncated");
  }
  std::vector<double> doubles(size_t n) {
    std::vector<double> v(n);
    bytes(v.data(), n * sizeof(double));
    return v;
  }
};

void check(int rc, const char* what) {
  if (rc != 0) {
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, ocfd_gpu_last_error());
    std::exit(2);  // the reference stops on its errors
  }
}

// one Fortran unformatted sequential record (gfortran: 4-byte length before and after)
void record(FILE* o, const void* p, int32_t n) {
  std::fwrite(&n, 4, 1, o);
  std::fwrite(p, 1, (size_t)n, o);
  std::fwrite(&n, 4, 1, o);
}
// write_3d (OCFD_IO_mpi.f90:232): one record of nx*ny doubles per k plane
void write_3d(FILE* o, const double* a, int nx, int ny, int nz) {
  for (int k = 0; k < nz; k++) record(o, a + (size_t)k * nx * ny, (int32_t)(sizeof(double) * nx * ny));
}

double sum(const std::vector<double>& v) {
  double s = 0.0;
  for (double x : v) s += x;
  return s;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s <case file> <output file> | --describe <case file>\n", argv[0]);
    return 1;
  }
  const bool describe = std::strcmp(argv[1], "--describe") == 0;
  const char* case_path = describe ? argv[2] : argv[1];
  ocfd_params P{};
  ocfd_thermo th{};
  ocfd_kinetics kin{};
  ocfd_transport tr{};
  ocfd_bcdata bc{};
  double dt = 0.0;
  int nsteps = 0, if_reaction = 0, nsub = 1, has_kin = 0, has_bc = 0, ns = 0, nfilt = 0, nana = 0;
  std::vector<double> coords, prim5, di, inlet, upper, wall, tm, fait;
  std::vector<double> filter(1000, 0.0), ana(1000, 0.0);  // Para%Filter, Para%ANA_Para (100 x 10)
  try {
    Reader r(case_path);
    if (!r.f) throw std::string("cannot open ") + case_path;
    char magic[8];
    r.bytes(magic, 8);
    if (std::memcmp(magic, "OCFDCASE", 8) != 0) throw std::string("not a case file");
    const int32_t version = r.get<int32_t>();
    if (version != 1 && version != 2) throw std::string("unknown case file version");
    const int32_t sp = r.get<int32_t>(), st = r.get<int32_t>(), sk = r.get<int32_t>(), str = r.get<int32_t>();
    if (sp != (int)sizeof P || st != (int)sizeof th || sk != (int)sizeof kin || str != (int)sizeof tr)
      throw std::string("record sizes differ from include/ocfd_gpu.h");
    r.bytes(&P, sizeof P);
    r.bytes(&th, sizeof th);
    has_kin = r.get<int32_t>();
    if (has_kin) r.bytes(&kin, sizeof kin);
    r.bytes(&tr, sizeof tr);
    dt = r.get<double>();
    nsteps = r.get<int32_t>();
    if_reaction = r.get<int32_t>();
    nsub = r.get<int32_t>();
    const int64_t H = r.get<int64_t>();
    coords = r.doubles(3 * (size_t)H);
    const int64_t N = r.get<int64_t>();
    prim5 = r.doubles(5 * (size_t)N);
    ns = r.get<int32_t>();
    di = r.doubles((size_t)ns * N);
    has_bc = r.get<int32_t>();
    if (has_bc) {
      std::vector<double>* arr[5] = {&inlet, &upper, &wall, &tm, &fait};
      for (auto* a : arr) *a = r.doubles((size_t)r.get<int64_t>());
      bc.inlet = inlet.empty() ? nullptr : inlet.data();
      bc.upper = upper.empty() ? nullptr : upper.data();
      bc.wall_pertb = wall.empty() ? nullptr : wall.data();
      bc.n_tm = (int)tm.size();
      bc.tm = tm.empty() ? nullptr : tm.data();
      bc.fait = fait.empty() ? nullptr : fait.data();
    }
    if (version >= 2) {  // NFiltering + Filter, ANA_Number + ANA_Para
      nfilt = r.get<int32_t>();
      r.bytes(filter.data(), sizeof(double) * 1000);
      nana = r.get<int32_t>();
      r.bytes(ana.data(), sizeof(double) * 1000);
      if (nfilt < 0 || nfilt > 10 || nana < 0 || nana > 10) throw std::string("NFiltering / ANA_Number must be 0..10");
    }
  } catch (const std::string& e) {
    std::fprintf(stderr, "%s\n", e.c_str());
    return 1;
  }

  if (describe) {
    std::printf("nx=%d ny=%d nz=%d lap=%d n_spec=%d nsteps=%d if_reaction=%d nsub=%d dt=%.17g kinetics=%d bc=%d "
                "n_tm=%d sum_coords=%.17g sum_prim=%.17g sum_di=%.17g nfiltering=%d ana_number=%d\n",
                P.nx, P.ny, P.nz, P.lap, ns, nsteps, if_reaction, nsub, dt, has_kin, has_bc, bc.n_tm,
                sum(coords), sum(prim5), sum(di), nfilt, nana);
    return 0;
  }
  // init3d + comput_flow_variables + OCFD_bc (OCFD_NS_Solver.f90:15-18)
  check(ocfd_gpu_init(&P, &th, has_kin ? &kin : nullptr, &tr, has_bc ? &bc : nullptr, coords.data(), nullptr),
        "ocfd_gpu_init");
  check(ocfd_gpu_init_state(prim5.data(), di.data(), 0.0), "ocfd_gpu_init_state");
  const long long N = (long long)P.nx * P.ny * P.nz;
  const long long H = (long long)(P.nx + 2 * P.lap) * (P.ny + 2 * P.lap) * (P.nz + 2 * P.lap);
  enum { ANA_TIME_AVERAGE = 100, ANA_Q = 101, ANA_BOX = 102 };  // MODULE_parameter.f90:28-29
  for (int m = 0; m < nana; m++)
    if (std::lround(ana[100 * m]) == ANA_BOX) check(ocfd_gpu_keep_viscosity(1), "ocfd_gpu_keep_viscosity");
  const int show = P.istep_show > 0 ? P.istep_show : 1;
  double tt = 0.0;
  std::vector<double> qbuf, abuf;
  for (int istep = 1; istep <= nsteps; istep++) {
    check(ocfd_gpu_flow_advance(0.5 * dt, tt), "flow_time_advance");                 // :28
    if (if_reaction) check(ocfd_gpu_chem_advance(dt / nsub, nsub), "Chemical_time_advance");  // :30-35
    check(ocfd_gpu_flow_advance(0.5 * dt, tt), "flow_time_advance");                 // :37
    tt = tt + dt;
    if (nfilt > 0) check(ocfd_gpu_filtering(istep, nfilt, filter.data(), nullptr), "filtering");  // :48
    if (istep % show == 0) {  // show_flow_msg (:50-52)
      double e = 0.0, k = 0.0;
      check(ocfd_gpu_diag(&e, &k), "show_flow_msg");
      std::printf("Istep=%d  tt=%.9e  E_mean=%.15e  K_mean=%.15e\n", istep, tt, e, k);
    }
    for (int m = 0; m < nana; m++) {  // OCFD_analysis (:55, OCFD_ANA.f90:3-33)
      const long kind = std::lround(ana[100 * m]), kstep = std::lround(ana[100 * m + 1]);
      if (kstep < 1 || istep % kstep != 0) continue;
      char name[64];
      if (kind == ANA_BOX) {
        double row[19];
        check(ocfd_gpu_ana_box(tt, row), "ana_box");
        FILE* o = std::fopen("statistics.dat", "a");
        if (!o) return 1;
        for (double x : row) std::fprintf(o, "%20.12f", x);
        std::fprintf(o, "\n");
        std::fclose(o);
      } else if (kind == ANA_Q) {
        qbuf.resize((size_t)N);
        check(ocfd_gpu_ana_q(qbuf.data()), "ana_getQ");
        std::snprintf(name, sizeof name, "Q-%07d.dat", istep);
        FILE* o = std::fopen(name, "wb");
        if (!o) return 1;
        write_3d(o, qbuf.data(), P.nx, P.ny, P.nz);
        std::fclose(o);
      } else if (kind == ANA_TIME_AVERAGE) {
        int ka = 0;
        double ta = 0.0;
        check(ocfd_gpu_ana_time_average(dt, &ka, &ta), "ana_time_average");
        const long ksave = std::lround(ana[100 * m + 2]);
        if (ksave >= 1 && istep % ksave == 0) {
          abuf.resize((size_t)(5 + ns) * N);
          check(ocfd_gpu_ana_average(0, abuf.data(), &ka, &ta), "ana_time_average");
          std::snprintf(name, sizeof name, "OCFD-comb%08d.dat.average", istep);
          FILE* o = std::fopen(name, "wb");
          if (!o) return 1;
          struct __attribute__((packed)) { int32_t k; double t; } hdr{ka, ta};
          record(o, &hdr, (int32_t)sizeof hdr);
          for (int f = 0; f < 5 + ns; f++) write_3d(o, abuf.data() + (size_t)f * N, P.nx, P.ny, P.nz);
          std::fclose(o);
        }
      } else {
        std::fprintf(stderr, "analysis kind %ld is not built\n", kind);
        return 2;
      }
    }
  }
  // save_flow_data: f, di and the seven primitives with their halos
  std::vector<double> fo(5 * N), dio((size_t)ns * H), pro(7 * H);
  check(ocfd_gpu_download_state(fo.data(), dio.data(), pro.data()), "ocfd_gpu_download_state");
  check(ocfd_gpu_finalize(), "ocfd_gpu_finalize");
  FILE* o = std::fopen(argv[2], "wb");
  if (!o) return 1;
  bool ok = std::fwrite(fo.data(), sizeof(double), fo.size(), o) == fo.size() &&
            std::fwrite(dio.data(), sizeof(double), dio.size(), o) == dio.size() &&
            std::fwrite(pro.data(), sizeof(double), pro.size(), o) == pro.size();
  std::fclose(o);
  return ok ? 0 : 1;
}
