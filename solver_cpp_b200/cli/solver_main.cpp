// `Solver`: command-line drop-in for the reference program (main.cpp:6-30)
// running every Krylov method on the B200 through the C ABI.
//
// Same flags (collection::readCMD, solver_collection.cpp:278-307) and defaults
// (solver_collection.cpp:26-49), the same input layout
// <CRS_Path>/<L1_Dir_Name>/<CRS_Dir_Name>/<CRS_Matrix_Name>/{ColVal,Ptr,bx}.txt
// (solver_collection.cpp:400-470), the same outputs ./output/<NAME>_his.txt
// and ./output/<NAME>_xvec.txt (cg.cpp:187-192,255-257) and the same summary
// lines ("|b-ax|2/|b|2 =", "loop =", "time =", "converge" / "not converge",
// cg.cpp:244-247, outerMethods.cpp:74-81). -c, -x, -t are accepted for
// compatibility: the solve always runs on the GPU and vectors never leave it.
// Added options: --precision fp64|fp32|bf16 (inner solve of VP methods),
// --reference-defects, --device N.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <fstream>
#include <map>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "krylov_sm100.h"

namespace {

struct Opt {
  std::string l1 = "Matrix", crs_path = "../", crs_dir = "CRS", crs_name = "NONE";
  std::string mm_path = "../", mm_dir = "MM", mm_name = "NONE";
  std::string outer = "", inner = "NO";
  int threads = 8;
  long long outer_maxloop = 10000, inner_maxloop = 50;
  double outer_eps = 1e-8, inner_eps = 1e-1;
  long long outer_restart = 1000, inner_restart = 1000;
  int outer_kskip = 2, inner_kskip = 2, outer_fix = 2, inner_fix = 2;
  bool verbose = false, cuda = false, pinned = false, multigpu = false;
  std::string precision = "fp64";
  bool reference_defects = false;
  int device = 0;
};

const char *kUsage =
    "usage: Solver -S <method> -m <matrix> [options]\n"
    "  -N --L1_Dir_Name (Matrix)  -p --CRS_Path (../)  -d --CRS_Dir_Name (CRS)  -m --CRS_Matrix_Name\n"
    "  -P --MM_Path (../)  -D --MM_Dir_Name (MM)  -M --MM_Matrix_Name: <P>/<N>/<D>/<M>/<M>.mtx, b = A*1\n"
    "  -t --Openmp_Thread (8, unused on GPU)\n"
    "  -S --OuterSolver  -L --OuterMaxLoop (10000)  -E --OuterEps (1e-8)  -R --OuterRestart (1000)\n"
    "  -K --OuterKskip (2)  -F --OuterFix (2)\n"
    "  -s --InnerSolver  -l --InnerMaxLoop (50)  -e --InnerEps (1e-1)  -r --InnerRestart (1000)\n"
    "  -k --InnerKskip (2)  -f --InnerFix (2)\n"
    "  -v --verbose  -c --cuda  -x --pinned  -g --multiGPU\n"
    "  --precision fp64|fp32|bf16  (inner solve of VP methods)  --reference-defects  --device N\n"
    "methods: cg bicg cr gcr gmres kskipcg kskipcr kskipbicg vpcg vpbicg vpcr vpgcr vpgmres\n";

// The times report (times::showTimeOnCPU / showTimeOnGPU, times.cpp:44-76),
// line for line, the format data2csv.sh parses. No host thread does Krylov
// arithmetic here, so the CPU block is zero; the GPU block holds the device
// time of each kernel class (ks_report.t_*): SpMVs with their fused
// epilogues, reductions (dots, norms, Gram and block dots, with the vector
// updates fused into them), memsets, and the copies of b in and x out.
void print_times(const ks_report &rep) {
  const double total = rep.solve_seconds > 0 ? rep.solve_seconds : 1e-30;
  auto line = [&](const char *label, double t) {
    std::cout << label << std::setprecision(6) << t << ", " << std::setprecision(2) << t / total * 100 << "%"
              << std::endl;
  };
  std::cout << "Execution time on CPU" << std::endl;
  line("\tDot process time = ", 0.0);
  line("\tMV process time  = ", 0.0);
  line("\t  cons time    = ", 0.0);
  line("\t  dis time    = ", 0.0);
  const double all = rep.t_mv + rep.t_dot;
  std::cout << "Execution time on GPU" << std::endl;
  line("\tDot process time  = ", rep.t_dot);
  line("\tMV process time   = ", rep.t_mv);
  line("\t  H2D time       = ", rep.t_h2d);
  line("\t  D2H time       = ", rep.t_d2h);
  line("\t  Memset time    = ", rep.t_memset);
  line("\tother time       = ", total - all);
  line("\t  Copy time    = ", 0.0);
  line("\t  cons time    = ", 0.0);
  line("\t  dis time    = ", 0.0);
}

// solver_collection.cpp:240-267
ks_solver to_solver(const std::string &s) {
  static const std::map<std::string, ks_solver> m = {
      {"cg", KS_CG},         {"CG", KS_CG},           {"bicg", KS_BICG},         {"BICG", KS_BICG},
      {"cr", KS_CR},         {"CR", KS_CR},           {"gcr", KS_GCR},           {"GCR", KS_GCR},
      {"gmres", KS_GMRES},   {"GMRES", KS_GMRES},     {"kskipcg", KS_KSKIPCG},   {"KSKIPCG", KS_KSKIPCG},
      {"kskipcr", KS_KSKIPCR}, {"KSKIPCR", KS_KSKIPCR}, {"kskipbicg", KS_KSKIPBICG}, {"KSKIPBICG", KS_KSKIPBICG},
      {"vpcg", KS_VPCG},     {"VPCG", KS_VPCG},       {"vpbicg", KS_VPBICG},     {"VPBICG", KS_VPBICG},
      {"vpcr", KS_VPCR},     {"VPCR", KS_VPCR},       {"vpgcr", KS_VPGCR},       {"VPGCR", KS_VPGCR},
      {"vpgmres", KS_VPGMRES}, {"VPGMRES", KS_VPGMRES}};
  auto it = m.find(s);
  return it == m.end() ? KS_NONE : it->second;
}

// solver_collection.cpp:205-238
const char *solver_name(ks_solver s) {
  static const char *names[] = {"NONE",    "CG",   "BICG",   "CR",   "GCR",   "GMRES",  "KSKIPCG",
                                "KSKIPCR", "KSKIPBICG", "VPCG", "VPBICG", "VPCR", "VPGCR", "VPGMRES"};
  return (s >= 0 && s <= 13) ? names[s] : "NONE";
}

[[noreturn]] void die(const std::string &msg, int code = -1) {
  std::cerr << msg << std::endl;
  std::exit(code);
}

bool parse(int argc, char **argv, Opt &o) {
  // short name -> long name
  static const std::map<std::string, std::string> alias = {
      {"-N", "L1_Dir_Name"},  {"-p", "CRS_Path"},     {"-d", "CRS_Dir_Name"},   {"-m", "CRS_Matrix_Name"},
      {"-P", "MM_Path"},      {"-D", "MM_Dir_Name"},  {"-M", "MM_Matrix_Name"}, {"-t", "Openmp_Thread"},
      {"-S", "OuterSolver"},  {"-L", "OuterMaxLoop"}, {"-E", "OuterEps"},       {"-R", "OuterRestart"},
      {"-K", "OuterKskip"},   {"-F", "OuterFix"},     {"-s", "InnerSolver"},    {"-l", "InnerMaxLoop"},
      {"-e", "InnerEps"},     {"-r", "InnerRestart"}, {"-k", "InnerKskip"},     {"-f", "InnerFix"},
      {"-v", "verbose"},      {"-c", "cuda"},         {"-x", "pinned"},         {"-g", "multiGPU"}};
  static const std::map<std::string, bool> is_flag = {{"verbose", true},  {"cuda", true},
                                                      {"pinned", true},   {"multiGPU", true},
                                                      {"reference-defects", true}, {"help", true}};
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    std::string key, val;
    bool has_val = false;
    if (a.rfind("--", 0) == 0) {
      key = a.substr(2);
      const size_t eq = key.find('=');
      if (eq != std::string::npos) {
        val = key.substr(eq + 1);
        key = key.substr(0, eq);
        has_val = true;
      }
    } else if (a.size() >= 2 && a[0] == '-') {
      auto it = alias.find(a.substr(0, 2));
      if (it == alias.end()) die("unknown option " + a + "\n" + kUsage);
      key = it->second;
      if (a.size() > 2) {
        val = a.substr(2);
        has_val = true;
      }
    } else {
      die("unexpected argument " + a + "\n" + kUsage);
    }
    if (key == "help") {
      std::cout << kUsage;
      std::exit(0);
    }
    static const char *known[] = {"L1_Dir_Name", "CRS_Path",     "CRS_Dir_Name", "CRS_Matrix_Name", "MM_Path",
                                  "MM_Dir_Name", "MM_Matrix_Name", "Openmp_Thread", "OuterSolver", "OuterMaxLoop",
                                  "OuterEps",    "OuterRestart", "OuterKskip",   "OuterFix",        "InnerSolver",
                                  "InnerMaxLoop", "InnerEps",    "InnerRestart", "InnerKskip",      "InnerFix",
                                  "verbose",     "cuda",         "pinned",       "multiGPU",        "precision",
                                  "reference-defects", "device"};
    bool ok = false;
    for (const char *k : known) ok = ok || key == k;
    if (!ok) die("unknown option --" + key + "\n" + kUsage);
    const bool flag = is_flag.count(key) > 0;
    if (!flag && !has_val) {
      if (i + 1 >= argc) die("option --" + key + " needs a value\n" + kUsage);
      val = argv[++i];
    }
    try {
      if (key == "L1_Dir_Name") o.l1 = val;
      else if (key == "CRS_Path") o.crs_path = val;
      else if (key == "CRS_Dir_Name") o.crs_dir = val;
      else if (key == "CRS_Matrix_Name") o.crs_name = val;
      else if (key == "MM_Path") o.mm_path = val;
      else if (key == "MM_Dir_Name") o.mm_dir = val;
      else if (key == "MM_Matrix_Name") o.mm_name = val;
      else if (key == "Openmp_Thread") o.threads = std::stoi(val);
      else if (key == "OuterSolver") o.outer = val;
      else if (key == "OuterMaxLoop") o.outer_maxloop = std::stoll(val);
      else if (key == "OuterEps") o.outer_eps = std::stod(val);
      else if (key == "OuterRestart") o.outer_restart = std::stoll(val);
      else if (key == "OuterKskip") o.outer_kskip = std::stoi(val);
      else if (key == "OuterFix") o.outer_fix = std::stoi(val);
      else if (key == "InnerSolver") o.inner = val;
      else if (key == "InnerMaxLoop") o.inner_maxloop = std::stoll(val);
      else if (key == "InnerEps") o.inner_eps = std::stod(val);
      else if (key == "InnerRestart") o.inner_restart = std::stoll(val);
      else if (key == "InnerKskip") o.inner_kskip = std::stoi(val);
      else if (key == "InnerFix") o.inner_fix = std::stoi(val);
      else if (key == "verbose") o.verbose = true;
      else if (key == "cuda") o.cuda = true;
      else if (key == "pinned") o.pinned = true;
      else if (key == "multiGPU") o.multigpu = true;
      else if (key == "precision") o.precision = val;
      else if (key == "reference-defects") o.reference_defects = true;
      else if (key == "device") o.device = std::stoi(val);
      else die("unknown option --" + key + "\n" + kUsage);
    } catch (const std::exception &) {
      die("bad value for --" + key + ": " + val);
    }
  }
  return true;
}

bool is_dir(const std::string &p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

}  // namespace

int main(int argc, char **argv) {
  Opt o;
  parse(argc, argv, o);
  // collection::readCMD checks (solver_collection.cpp:344-378)
  if (o.outer.empty()) die(std::string("[X]OuterSolver (-S) is required\n") + kUsage);
  if (o.mm_name == "NONE" && o.crs_name == "NONE") die("[X]Must set one input source");
  if (o.mm_name != "NONE" && o.crs_name != "NONE") die("[X]Only can set one input source");
  const ks_solver outer = to_solver(o.outer);
  if (outer == KS_NONE) die("[X]OuterSolverName can not found in List");
  const ks_solver inner = o.inner == "NO" ? KS_NONE : to_solver(o.inner);
  if (o.inner != "NO" && inner == KS_NONE) die("[X]InnerSolverName can not found in List");
  if (o.multigpu) die("Number of CUDA Device is less than 2, Can not Enable MultiGPU Mode");
  ks_precision prec = KS_FP64;
  if (o.precision == "fp32") prec = KS_FP32;
  else if (o.precision == "bf16") prec = KS_BF16;
  else if (o.precision != "fp64") die("--precision must be fp64, fp32 or bf16");

  int64_t n = 0, nnz = 0;
  std::vector<int32_t> ptr, col;
  std::vector<double> val, b, x;
  if (o.crs_name != "NONE") {
    // collection::checkCMD / checkCRSMatrix / readMatrix (solver_collection.cpp:391-828)
    const std::string dir = o.crs_path + "/" + o.l1 + "/" + o.crs_dir + "/" + o.crs_name;
    if (!is_dir(dir)) die("[X]Error no CRS files Dir -> " + dir);
    if (ks_crs_read_header(dir.c_str(), &n, &nnz) != KS_OK)
      die("[X] Error in CRS files (missing, or N / M / NNZ differ between ColVal.txt, Ptr.txt, bx.txt, or N != M)");
    ptr.resize((size_t)n + 1);
    col.resize((size_t)nnz);
    val.resize((size_t)nnz);
    b.resize((size_t)n);
    x.resize((size_t)n);
    if (ks_crs_read(dir.c_str(), n, nnz, ptr.data(), col.data(), val.data(), b.data(), x.data()) != KS_OK)
      die("[X] Read CRS files fail");
  } else {
    // Matrix Market source, laid out as the reference checks it
    // (solver_collection.cpp:505-601): <P>/<N>/<D>/<M>/<M>.mtx. The file
    // holds no right-hand side: b = A * (1, ..., 1), x0 = 0.
    const std::string dir = o.mm_path + "/" + o.l1 + "/" + o.mm_dir + "/" + o.mm_name;
    if (!is_dir(dir)) die("[X]Error no MM files Dir -> " + dir);
    const std::string file = dir + "/" + o.mm_name + ".mtx";
    const ks_status hs = ks_mm_read_header(file.c_str(), &n, &nnz);
    if (hs != KS_OK) die("[X]Error in mm file " + file + ": " + ks_status_string(hs));
    ptr.resize((size_t)n + 1);
    col.resize((size_t)std::max<int64_t>(nnz, 1));
    val.resize((size_t)std::max<int64_t>(nnz, 1));
    if (ks_mm_read(file.c_str(), n, nnz, ptr.data(), col.data(), val.data()) != KS_OK)
      die("[X] Read mm file fail");
    b.assign((size_t)n, 0.0);
    x.assign((size_t)n, 0.0);
    for (int64_t i = 0; i < n; i++)
      for (int32_t j = ptr[(size_t)i]; j < ptr[(size_t)i + 1]; j++) b[(size_t)i] += val[(size_t)j];
  }

  const bool vp = outer == KS_VPCG || outer == KS_VPCR || outer == KS_VPGCR || outer == KS_VPGMRES ||
                  outer == KS_VPBICG;
  // collection::showCMD (solver_collection.cpp:603-652), the lines
  // data2csv.sh reads ("CUDA :", "MultiGPU :") among them; this program
  // always runs on the GPU, on one device
  std::cout << "=========================================================" << std::endl;
  std::cout << "InputSource : " << (o.crs_name != "NONE" ? "CRS" : "MM") << std::endl;
  std::cout << "FullPath : "
            << (o.crs_name != "NONE" ? o.crs_path + "/" + o.l1 + "/" + o.crs_dir + "/" + o.crs_name
                                     : o.mm_path + "/" + o.l1 + "/" + o.mm_dir + "/" + o.mm_name)
            << std::endl;
  std::cout << "N : " << n << std::endl;
  std::cout << "NNZ : " << nnz << std::endl;
  std::cout << "-------------" << std::endl;
  std::cout << "OpenMP thread : " << o.threads << std::endl;
  std::cout << "GPU Num : " << o.device << std::endl;
  std::cout << "-------------" << std::endl;
  std::cout << "VP : " << (vp ? "On" : "Off") << std::endl;
  std::cout << "CUDA : On" << std::endl;
  std::cout << "Pinned : " << (o.pinned ? "On" : "Off") << std::endl;
  std::cout << "MultiGPU : Off" << std::endl;
  std::cout << "-------------" << std::endl;
  std::cout << "OuterSolver : " << solver_name(outer) << std::endl;
  std::cout << "OuterMaxLoop : " << o.outer_maxloop << std::endl;
  std::cout << "OuterEps : " << o.outer_eps << std::endl;
  std::cout << "OuterRestart : " << o.outer_restart << std::endl;
  std::cout << "OuterKskip : " << o.outer_kskip << std::endl;
  std::cout << "OuterFix : " << o.outer_fix << std::endl;
  std::cout << "-------------" << std::endl;
  std::cout << "InnerSolver : " << solver_name(inner) << std::endl;
  std::cout << "InnerMaxLoop : " << o.inner_maxloop << std::endl;
  std::cout << "InnerEps : " << o.inner_eps << std::endl;
  std::cout << "InnerRestart : " << o.inner_restart << std::endl;
  std::cout << "InnerKskip : " << o.inner_kskip << std::endl;
  std::cout << "InnerFix : " << o.inner_fix << std::endl;
  std::cout << "=========================================================" << std::endl;
  if (outer == KS_KSKIPCR || outer == KS_VPBICG) {  // outerMethods.cpp:46-48,57-59
    std::cout << "Not implemented" << std::endl;
    std::cerr << "outer result -> 99" << std::endl;
    return 0;
  }

  ks_ctx *ctx = nullptr;
  ks_status s = ks_ctx_create(o.device, &ctx);
  if (s != KS_OK) die(std::string("[X]CUDA device: ") + ks_status_string(s), 1);
  const bool needT = outer == KS_BICG || outer == KS_KSKIPBICG || (vp && (inner == KS_BICG || inner == KS_KSKIPBICG));
  unsigned flags = needT ? KS_MAT_TRANSPOSE : 0u;
  if (vp && prec == KS_FP32) flags |= KS_MAT_FP32;
  if (vp && prec == KS_BF16) flags |= KS_MAT_BF16;
  ks_mat *A = nullptr;
  s = ks_csr_upload(ctx, n, nnz, ptr.data(), col.data(), val.data(), flags, &A);
  if (s != KS_OK) die(std::string("[X]upload: ") + ks_status_string(s) + " " + ks_last_error(ctx), 1);

  ks_params p;
  ks_params_default(&p);
  p.outer_maxloop = o.outer_maxloop;
  p.outer_eps = o.outer_eps;
  p.outer_restart = o.outer_restart;
  p.outer_kskip = o.outer_kskip;
  p.outer_fix = o.outer_fix;
  p.inner_maxloop = o.inner_maxloop;
  p.inner_eps = o.inner_eps;
  p.inner_restart = o.inner_restart;
  p.inner_kskip = o.inner_kskip;
  p.inner_fix = o.inner_fix;
  p.inner_precision = prec;
  p.reference_defects = o.reference_defects ? 1 : 0;
  p.profile = 1;  // the times report below
  const int64_t cap = o.outer_maxloop + 2;
  std::vector<int64_t> hit((size_t)cap);
  std::vector<double> herr((size_t)cap);
  ks_report rep;
  std::memset(&rep, 0, sizeof(rep));
  const ks_status r = ks_solve_host(ctx, A, outer, inner, &p, b.data(), x.data(), hit.data(), herr.data(), cap, &rep);
  if (!(r == KS_OK || r == KS_NOT_CONVERGED || r == KS_BREAKDOWN || r == KS_NAN_DETECTED)) {
    std::cerr << "outer result -> " << r << " (" << ks_status_string(r) << ": " << ks_last_error(ctx) << ")"
              << std::endl;
    std::cerr << "[X]Some Error in methods" << std::endl;
    ks_mat_destroy(A);
    ks_ctx_destroy(ctx);
    return 1;
  }

  mkdir("./output", 0755);
  const std::string nm = solver_name(outer);
  {
    std::ofstream his("./output/" + nm + "_his.txt");
    if (!his.is_open()) die("File open error");
    const int64_t m = std::min<int64_t>(rep.hist_len, cap);
    for (int64_t i = 0; i < m; i++) {
      if (o.verbose)
        std::cout << hit[i] << " " << std::scientific << std::setprecision(12) << std::uppercase << herr[i]
                  << std::endl;
      his << hit[i] << " " << std::scientific << std::setprecision(12) << std::uppercase << herr[i] << "\n";
    }
  }
  std::cout << "|b-ax|2/|b|2 = " << std::fixed << std::setprecision(1) << rep.true_res_log10 << std::endl;
  std::cout << "loop = " << rep.loop << std::endl;
  std::cout << "time = " << std::setprecision(6) << rep.solve_seconds << std::endl;
  print_times(rep);
  std::cout << "true |b-Ax|/|b| = " << std::scientific << std::setprecision(3) << rep.true_rel_res << std::endl;
  {
    std::ofstream fx("./output/" + nm + "_xvec.txt");
    if (!fx.is_open()) die("File open error");
    for (int64_t i = 0; i < n; i++)
      fx << i << " " << std::scientific << std::setprecision(12) << std::uppercase << x[(size_t)i] << "\n";
  }
  if (r == KS_OK)
    std::cout << "converge" << std::endl;
  else
    std::cout << "not converge" << std::endl;
  ks_mat_destroy(A);
  ks_ctx_destroy(ctx);
  return 0;
}
