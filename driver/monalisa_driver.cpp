// monalisa_driver -- standalone CG-SENSE reconstruction through the C ABI of
// libmonalisa_gpu.so (include/monalisa_gpu.h), with no MATLAB and no Python.
//
// The chain is the one the reference's scripts run in MATLAB
// (bmTraj2SparseMat -> bmKF / bmKF_conj -> bmSensa):
//   mlg_traj2sparsemat3   Gu / Gut from the trajectory (src/gridding123/m/bmTraj2SparseMat.m)
//   mlg_deapodization     K (src/fourier123/prep_function/bmK.m), then on the host
//                         KFC = K / prod(N_u) / prod(dK_u) .* C   (bmKF.m:27-34)
//                         KFC_conj = K / prod(dK_u) .* conj(C)      (bmKF_conj.m:30-37)
//   mlg_plan_create, mlg_plan_set_dk
//   mlg_sensa             CG-SENSE (src/fourier123/solver_function/imDim/nonCartesian/bmSensa.m)
//
// Inputs come from .npy files (trajectory, volume elements, coil maps,
// k-space) or from a built-in synthetic workload (2-D golden-angle radial or
// 3-D phyllotaxis koosh ball, a disc/ball phantom, k-space simulated by the
// forward operator).  Options are given on the command line (--key value) or
// in a flat JSON object (--config file.json; command-line options override
// it).  The image is written as a complex64 .npy vector [prod(n_u)] (x
// fastest, the reference's column order); the residual history and timings
// are printed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "monalisa_gpu.h"

using cf = std::complex<float>;

namespace {

[[noreturn]] void die(const std::string& msg) {
  std::fprintf(stderr, "monalisa_driver: %s\n", msg.c_str());
  std::exit(2);
}

void check(int st, const char* what) {
  if (st != MLG_OK) die(std::string(what) + ": " + mlg_status_string(st) + ": " + mlg_last_error());
}

// ---- .npy files (little-endian, C order) ------------------------------------
struct Npy {
  std::string descr;
  std::vector<size_t> shape;
  std::vector<char> data;
  size_t count() const {
    size_t n = 1;
    for (size_t s : shape) n *= s;
    return n;
  }
};

Npy npy_read(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) die("cannot open " + path);
  char magic[6];
  f.read(magic, 6);
  if (std::memcmp(magic, "\x93NUMPY", 6) != 0) die(path + ": not a .npy file");
  unsigned char ver[2];
  f.read(reinterpret_cast<char*>(ver), 2);
  uint32_t hlen = 0;
  if (ver[0] == 1) {
    uint16_t h;
    f.read(reinterpret_cast<char*>(&h), 2);
    hlen = h;
  } else {
    f.read(reinterpret_cast<char*>(&hlen), 4);
  }
  std::string hdr(hlen, '\0');
  f.read(&hdr[0], hlen);
  Npy a;
  auto field = [&](const char* key) {
    const size_t k = hdr.find(key);
    if (k == std::string::npos) die(path + ": header lacks " + key);
    return hdr.substr(hdr.find(':', k) + 1);
  };
  std::string d = field("'descr'");
  const size_t q0 = d.find('\''), q1 = d.find('\'', q0 + 1);
  a.descr = d.substr(q0 + 1, q1 - q0 - 1);
  if (field("'fortran_order'").find("True") < field("'fortran_order'").find(','))
    die(path + ": Fortran-ordered arrays are not read (save with C order)");
  std::string s = field("'shape'");
  s = s.substr(s.find('(') + 1, s.find(')') - s.find('(') - 1);
  std::stringstream ss(s);
  std::string tok;
  while (std::getline(ss, tok, ','))
    if (tok.find_first_of("0123456789") != std::string::npos) a.shape.push_back(std::stoull(tok));
  size_t esz = a.descr == "<f8" || a.descr == "<c8" ? 8 : a.descr == "<f4" ? 4 : a.descr == "<c16" ? 16 : 0;
  if (!esz) die(path + ": unsupported dtype " + a.descr + " (float32, float64, complex64, complex128)");
  a.data.resize(a.count() * esz);
  f.read(a.data.data(), (std::streamsize)a.data.size());
  if (!f) die(path + ": truncated data");
  return a;
}

std::vector<double> npy_real(const Npy& a) {
  std::vector<double> v(a.count());
  for (size_t i = 0; i < v.size(); ++i) {
    if (a.descr == "<f8")
      v[i] = reinterpret_cast<const double*>(a.data.data())[i];
    else if (a.descr == "<f4")
      v[i] = reinterpret_cast<const float*>(a.data.data())[i];
    else
      die("expected a real array, got " + a.descr);
  }
  return v;
}

std::vector<cf> npy_complex(const Npy& a) {
  std::vector<cf> v(a.count());
  if (a.descr == "<f4" || a.descr == "<f8") {
    const std::vector<double> r = npy_real(a);
    for (size_t i = 0; i < v.size(); ++i) v[i] = cf((float)r[i], 0.f);
    return v;
  }
  for (size_t i = 0; i < v.size(); ++i) {
    if (a.descr == "<c8")
      v[i] = reinterpret_cast<const cf*>(a.data.data())[i];
    else if (a.descr == "<c16")
      v[i] = cf(reinterpret_cast<const std::complex<double>*>(a.data.data())[i]);
    else
      die("expected a complex array, got " + a.descr);
  }
  return v;
}

void npy_write_c64(const std::string& path, const std::vector<cf>& v) {
  std::string hdr = "{'descr': '<c8', 'fortran_order': False, 'shape': (" + std::to_string(v.size()) + ",), }";
  while ((10 + hdr.size() + 1) % 64) hdr += ' ';
  hdr += '\n';
  std::ofstream f(path, std::ios::binary);
  if (!f) die("cannot write " + path);
  f.write("\x93NUMPY\x01\x00", 8);
  const uint16_t h = (uint16_t)hdr.size();
  f.write(reinterpret_cast<const char*>(&h), 2);
  f.write(hdr.data(), (std::streamsize)hdr.size());
  f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(cf)));
}

// ---- options -------------------------------------------------------------------
// Flat JSON object: "key": number | "string" | [numbers] | true/false.
void json_read(const std::string& path, std::map<std::string, std::string>& opt) {
  std::ifstream f(path);
  if (!f) die("cannot open " + path);
  std::stringstream buf;
  buf << f.rdbuf();
  const std::string s = buf.str();
  size_t i = s.find('{');
  if (i == std::string::npos) die(path + ": not a JSON object");
  ++i;
  auto skip = [&] {
    while (i < s.size() && (std::isspace((unsigned char)s[i]) || s[i] == ',')) ++i;
  };
  for (;;) {
    skip();
    if (i >= s.size() || s[i] == '}') break;
    if (s[i] != '"') die(path + ": expected a key at offset " + std::to_string(i));
    const size_t k1 = s.find('"', i + 1);
    const std::string key = s.substr(i + 1, k1 - i - 1);
    i = s.find(':', k1) + 1;
    while (std::isspace((unsigned char)s[i])) ++i;
    std::string val;
    if (s[i] == '"') {
      const size_t e = s.find('"', i + 1);
      val = s.substr(i + 1, e - i - 1);
      i = e + 1;
    } else if (s[i] == '[') {
      const size_t e = s.find(']', i);
      val = s.substr(i + 1, e - i - 1);
      val.erase(std::remove_if(val.begin(), val.end(), [](char c) { return std::isspace((unsigned char)c); }),
                val.end());
      i = e + 1;
    } else {
      const size_t e = s.find_first_of(",}", i);
      val = s.substr(i, e - i);
      while (!val.empty() && std::isspace((unsigned char)val.back())) val.pop_back();
      i = e;
    }
    opt[key] = val;
  }
}

std::vector<double> numbers(const std::string& s) {
  std::vector<double> v;
  std::stringstream ss(s);
  std::string tok;
  while (std::getline(ss, tok, ','))
    if (!tok.empty()) v.push_back(std::stod(tok));
  return v;
}

const char* kUsage =
    "usage: monalisa_driver [--config cfg.json] [--key value ...]\n"
    "  workload: --synthetic radial2d|koosh3d (with --n, --spokes, --samples, --coils)\n"
    "            or --traj t.npy --ve ve.npy --kspace y.npy [--coils_file C.npy] --N ... --n ...\n"
    "  t.npy [imDim, nPt] float64 (physical units), ve.npy [nPt], y.npy [nPt, nCh] complex64,\n"
    "  C.npy [prod(n_u), nCh] complex64 (x fastest); default C = 1\n"
    "  --N 512,512  --n 256,256  --dK 1,1  --kernel gauss|kaiser  --nWin 3  --kernelParam 0.61,10\n"
    "  --nIter 1  --nCGD 20  --ve_max 0 (0: max(ve))  --device 0  --repeat 1  --out x.npy\n"
    "  --dry-run: print the resolved options and exit (no device use)\n";

// ---- synthetic workloads -----------------------------------------------------
struct Workload {
  int imDim = 2;
  std::vector<int> N, n;
  std::vector<double> t;   // [nPt][imDim] (column-major [imDim, nPt])
  std::vector<float> ve;   // [nPt]
  std::vector<cf> C;       // [nu][nCh]
  std::vector<cf> y;       // [nPt][nCh]
  int nPt = 0, nCh = 1;
  std::vector<cf> phantom;  // synthetic only
};

const double kGolden = (1.0 + std::sqrt(5.0)) / 2.0;

// 2-D radial, spoke k at k*180deg/golden ratio, radii (-N/2 .. N/2-1) kMax/(N/2)
void golden_radial2(int nRead, int nSpoke, double dK_n, std::vector<double>& t) {
  const double kMax = nRead * dK_n / 2;
  t.resize(2 * (size_t)nRead * nSpoke);
  for (int s = 0; s < nSpoke; ++s) {
    const double phi = s * M_PI / kGolden;
    for (int r = 0; r < nRead; ++r) {
      const double rad = (r - nRead / 2) * kMax / (nRead / 2);
      const size_t p = (size_t)s * nRead + r;
      t[2 * p] = rad * std::cos(phi);
      t[2 * p + 1] = rad * std::sin(phi);
    }
  }
}

// 3-D koosh ball: spiral phyllotaxis directions (src/traj3/bmPhyllotaxisAngle3.m,
// one shot), lines of nRead samples at (-1/2 .. 1/2 - 1/nRead) nRead dK_n
void koosh3(int nRead, int nSpoke, double dK_n, std::vector<double>& t) {
  const double golden_angle = 2 * M_PI - 2 * M_PI / kGolden;
  const double q = M_PI / (2 * std::sqrt((double)nSpoke));
  t.resize(3 * (size_t)nRead * nSpoke);
  for (int s = 0; s < nSpoke; ++s) {
    const double counter = s + 1;
    const double phi = std::fmod(counter * golden_angle, 2 * M_PI), theta = q * std::sqrt(counter);
    for (int r = 0; r < nRead; ++r) {
      const double rad = (-0.5 + (double)r / nRead) * nRead * dK_n;
      const size_t p = (size_t)s * nRead + r;
      t[3 * p] = rad * std::cos(phi) * std::sin(theta);
      t[3 * p + 1] = rad * std::sin(phi) * std::sin(theta);
      t[3 * p + 2] = rad * std::cos(theta);
    }
  }
}

void synthetic(const std::string& kind, std::map<std::string, std::string>& opt, Workload& w) {
  auto geti = [&](const char* k, int def) { return opt.count(k) ? std::atoi(opt[k].c_str()) : def; };
  const bool d3 = kind == "koosh3d";
  if (!d3 && kind != "radial2d") die("unknown synthetic workload '" + kind + "' (radial2d, koosh3d)");
  w.imDim = d3 ? 3 : 2;
  const int n = geti("n", d3 ? 64 : 256), Ng = 2 * n;
  const int nRead = geti("samples", d3 ? 2 * n : 2 * n), nSpoke = geti("spokes", d3 ? 1024 : 256);
  w.nCh = geti("coils", d3 ? 8 : 1);
  w.N.assign(w.imDim, Ng);
  w.n.assign(w.imDim, n);
  if (d3)
    koosh3(nRead, nSpoke, (double)Ng / nRead, w.t);
  else
    golden_radial2(nRead, nSpoke, (double)Ng / nRead, w.t);
  w.nPt = nRead * nSpoke;
  if (!opt.count("kernel")) opt["kernel"] = d3 ? "gauss" : "kaiser";
  if (!opt.count("kernelParam")) opt["kernelParam"] = d3 ? "0.61,10" : "1.95,10,10";
  // volume elements of the radial lines on the device (device trajectory [imDim][nPt])
  std::vector<double> trow((size_t)w.imDim * w.nPt);
  for (int p = 0; p < w.nPt; ++p)
    for (int d = 0; d < w.imDim; ++d) trow[(size_t)d * w.nPt + p] = w.t[(size_t)p * w.imDim + d];
  double *dt = nullptr, *dv = nullptr;
  if (cudaMalloc(&dt, trow.size() * 8) != cudaSuccess || cudaMalloc(&dv, (size_t)w.nPt * 8) != cudaSuccess)
    die("device allocation failed");
  cudaMemcpy(dt, trow.data(), trow.size() * 8, cudaMemcpyHostToDevice);
  check(mlg_volume_element_radial_dev(w.imDim, w.nPt, nRead, dt, dv, nullptr), "mlg_volume_element_radial_dev");
  std::vector<double> ve(w.nPt);
  cudaMemcpy(ve.data(), dv, (size_t)w.nPt * 8, cudaMemcpyDeviceToHost);
  cudaFree(dt);
  cudaFree(dv);
  w.ve.assign(ve.begin(), ve.end());
  // smooth coil maps: Gaussian profiles around coils on a ring, linear phase
  long long nu = 1;
  for (int v : w.n) nu *= v;
  w.C.resize((size_t)nu * w.nCh);
  w.phantom.assign((size_t)nu, cf(0, 0));
  for (long long i = 0; i < nu; ++i) {
    double r[3] = {0, 0, 0};
    long long q = i;
    for (int d = 0; d < w.imDim; ++d) {
      r[d] = (double)(q % w.n[d]) / w.n[d] - 0.5;
      q /= w.n[d];
    }
    for (int c = 0; c < w.nCh; ++c) {
      const double a = 2 * M_PI * c / w.nCh;
      const double cx = 0.6 * std::cos(a), cy = 0.6 * std::sin(a), cz = d3 ? 0.3 * ((c & 1) ? 1 : -1) : 0;
      const double d2 = (r[0] - cx) * (r[0] - cx) + (r[1] - cy) * (r[1] - cy) + (r[2] - cz) * (r[2] - cz);
      const double mag = w.nCh == 1 ? 1.0 : std::exp(-d2 / 0.5);
      const double ph = w.nCh == 1 ? 0.0 : 2 * M_PI * (0.3 * r[0] * std::cos(a) + 0.3 * r[1] * std::sin(a));
      w.C[(size_t)i * w.nCh + c] = cf((float)(mag * std::cos(ph)), (float)(mag * std::sin(ph)));
    }
    const double rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    const double e = (r[0] - 0.1) * (r[0] - 0.1) / 0.02 + (r[1] + 0.05) * (r[1] + 0.05) / 0.01 + r[2] * r[2] / 0.02;
    w.phantom[i] = cf((float)((rr < 0.16 ? 1.0 : 0.0) + (e < 1 ? 0.5 : 0.0)), 0.f);
  }
}

}  // namespace

int main(int argc, char** argv) {
  std::map<std::string, std::string> opt;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a == "--help" || a == "-h") {
      std::fputs(kUsage, stdout);
      return 0;
    }
    if (a == "--dry-run") {
      opt["dry-run"] = "1";
      continue;
    }
    if (a.rfind("--", 0) != 0 || i + 1 >= argc) die("bad argument '" + a + "'\n" + kUsage);
    const std::string key = a.substr(2), val = argv[++i];
    if (key == "config") {
      std::map<std::string, std::string> cfg;
      json_read(val, cfg);
      for (auto& kv : cfg)
        if (!opt.count(kv.first)) opt[kv.first] = kv.second;
    } else {
      opt[key] = val;  // the command line overrides the file
    }
  }
  auto get = [&](const char* k, const char* def) { return opt.count(k) ? opt[k] : std::string(def); };
  if (opt.count("dry-run")) {
    for (auto& kv : opt) std::printf("%s = %s\n", kv.first.c_str(), kv.second.c_str());
    return 0;
  }
  check(mlg_set_device(std::atoi(get("device", "0").c_str())), "mlg_set_device");
  cudaSetDevice(std::atoi(get("device", "0").c_str()));

  Workload w;
  const bool synth = opt.count("synthetic") > 0;
  if (synth) {
    synthetic(opt["synthetic"], opt, w);
  } else {
    if (!opt.count("traj") || !opt.count("ve") || !opt.count("kspace") || !opt.count("N"))
      die(std::string("file mode needs --traj, --ve, --kspace and --N\n") + kUsage);
    Npy t = npy_read(opt["traj"]);
    if (t.shape.size() != 2 || t.shape[0] < 1 || t.shape[0] > 3) die("traj must be [imDim, nPt]");
    w.imDim = (int)t.shape[0];
    w.nPt = (int)t.shape[1];
    std::vector<double> tv = npy_real(t);
    w.t.resize(tv.size());
    for (int p = 0; p < w.nPt; ++p)
      for (int d = 0; d < w.imDim; ++d) w.t[(size_t)p * w.imDim + d] = tv[(size_t)d * w.nPt + p];
    std::vector<double> ve = npy_real(npy_read(opt["ve"]));
    if ((int)ve.size() != w.nPt) die("ve must have nPt values");
    w.ve.assign(ve.begin(), ve.end());
    Npy y = npy_read(opt["kspace"]);
    w.y = npy_complex(y);
    w.nCh = y.shape.size() == 2 ? (int)y.shape[1] : 1;
    if ((size_t)w.nPt * w.nCh != w.y.size()) die("kspace must be [nPt, nCh]");
    for (double v : numbers(opt["N"])) w.N.push_back((int)v);
    for (double v : numbers(get("n", opt["N"].c_str()))) w.n.push_back((int)v);
    if ((int)w.N.size() != w.imDim || (int)w.n.size() != w.imDim) die("--N / --n need imDim values");
  }
  long long nu = 1, Nu = 1;
  for (int d = 0; d < w.imDim; ++d) {
    nu *= w.n[d];
    Nu *= w.N[d];
  }
  if (!synth) {
    if (opt.count("coils_file")) {
      Npy c = npy_read(opt["coils_file"]);
      w.C = npy_complex(c);
      if ((long long)w.C.size() != nu * w.nCh) die("coil maps must be [prod(n_u), nCh]");
    } else {
      w.C.assign((size_t)nu * w.nCh, cf(1, 0));
    }
  }
  std::vector<double> dK = numbers(get("dK", ""));
  if (dK.empty()) dK.assign(w.imDim, 1.0);
  if ((int)dK.size() != w.imDim) die("--dK needs imDim values");
  const std::string kname = get("kernel", "gauss");
  const int ktype = kname == "kaiser" ? MLG_KERNEL_KAISER : MLG_KERNEL_GAUSS;
  const int nWin = std::atoi(get("nWin", "3").c_str());
  std::vector<double> kp = numbers(get("kernelParam", ktype == MLG_KERNEL_KAISER ? "1.95,10,10" : "0.61,10"));
  kp.resize(3, 0.0);
  for (double& v : kp) v = (double)(float)v;  // kernel parameters are single precision (bmVarargin_kernelType_nWin_kernelParam)
  // dK_u enters as single precision (the MATLAB wrappers' single(dK_u))
  std::vector<double> dKs(w.imDim);
  for (int d = 0; d < w.imDim; ++d) dKs[d] = (double)(float)dK[d];

  const auto t0 = std::chrono::steady_clock::now();
  mlg_matrix_t Gu = nullptr, Gut = nullptr;
  check(mlg_traj2sparsemat3(w.imDim, w.nPt, w.t.data(), nullptr, w.N.data(), dK.data(), ktype, nWin, kp.data(),
                            nullptr, &Gu, &Gut),
        "mlg_traj2sparsemat3");
  // K (one column), cropped to n_u; KFC and KFC_conj as bmKF / bmKF_conj, in
  // single precision: (K * F) * C with F = 1/prod(N_u)/prod(dK_u), resp. 1/prod(dK_u)
  std::vector<float> K((size_t)Nu);
  check(mlg_deapodization(w.imDim, w.N.data(), dKs.data(), ktype, nWin, kp.data(), K.data()), "mlg_deapodization");
  float pN = 1.f, pdK = 1.f;
  for (int d = 0; d < w.imDim; ++d) {
    pN *= (float)w.N[d];
    pdK *= (float)dKs[d];
  }
  const float F = (1.f / pN) / pdK, Fc = 1.f / pdK;
  std::vector<float> kr((size_t)nu * w.nCh), ki(kr.size()), cr(kr.size()), ci(kr.size());
  for (long long i = 0; i < nu; ++i) {
    long long q = i, cell = 0, stride = 1;
    for (int d = 0; d < w.imDim; ++d) {
      const long long x = q % w.n[d] + (w.N[d] / 2 - w.n[d] / 2);
      q /= w.n[d];
      cell += x * stride;
      stride *= w.N[d];
    }
    const float k = K[(size_t)cell], kf = k * F, kc = k * Fc;
    for (int c = 0; c < w.nCh; ++c) {
      const cf C = w.C[(size_t)i * w.nCh + c];
      const size_t o = (size_t)c * nu + i;  // column layout [prod(n_u), nCh]
      kr[o] = kf * C.real();
      ki[o] = kf * C.imag();
      cr[o] = kc * C.real();
      ci[o] = kc * -C.imag();
    }
  }
  mlg_plan_t plan = nullptr;
  check(mlg_plan_create(w.imDim, w.N.data(), w.n.data(), w.nCh, Gu, Gut, kr.data(), ki.data(), cr.data(), ci.data(),
                        &plan),
        "mlg_plan_create");
  check(mlg_plan_set_dk(plan, dKs.data()), "mlg_plan_set_dk");
  const double setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

  if (synth) {  // k-space of the phantom by the forward operator
    float2 *dx = nullptr, *dy = nullptr;
    if (cudaMalloc(&dx, (size_t)nu * 8) != cudaSuccess || cudaMalloc(&dy, (size_t)w.nPt * w.nCh * 8) != cudaSuccess)
      die("device allocation failed");
    cudaMemcpy(dx, w.phantom.data(), (size_t)nu * 8, cudaMemcpyHostToDevice);
    check(mlg_shanna_dev(plan, dx, 0, dy, nullptr), "mlg_shanna_dev");
    w.y.resize((size_t)w.nPt * w.nCh);
    if (cudaMemcpy(w.y.data(), dy, w.y.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess) die("copy failed");
    cudaFree(dx);
    cudaFree(dy);
  }
  // CG-SENSE with host buffers: y [nPt, nCh] column-major, x [prod(n_u)]
  std::vector<float> yR((size_t)w.nPt * w.nCh), yI(yR.size());
  for (int p = 0; p < w.nPt; ++p)
    for (int c = 0; c < w.nCh; ++c) {
      yR[(size_t)c * w.nPt + p] = w.y[(size_t)p * w.nCh + c].real();
      yI[(size_t)c * w.nPt + p] = w.y[(size_t)p * w.nCh + c].imag();
    }
  const int nIter = std::atoi(get("nIter", "1").c_str()), nCGD = std::atoi(get("nCGD", "20").c_str());
  const int repeat = std::max(1, std::atoi(get("repeat", "1").c_str()));
  const float ve_max = (float)std::atof(get("ve_max", "0").c_str());
  std::vector<float> xR((size_t)nu), xI((size_t)nu);
  std::vector<double> res(std::max(1, nIter));
  double best_ms = 1e300;
  for (int r = 0; r < repeat; ++r) {
    std::fill(xR.begin(), xR.end(), 0.f);
    std::fill(xI.begin(), xI.end(), 0.f);
    const auto a = std::chrono::steady_clock::now();
    check(mlg_sensa(plan, yR.data(), yI.data(), w.ve.data(), ve_max, nIter, nCGD, xR.data(), xI.data(), res.data()),
          "mlg_sensa");
    best_ms = std::min(best_ms, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count());
  }
  std::vector<cf> x((size_t)nu);
  for (long long i = 0; i < nu; ++i) x[i] = cf(xR[i], xI[i]);
  if (opt.count("out")) npy_write_c64(opt["out"], x);
  double err = -1;
  if (synth) {
    double num = 0, den = 0;
    for (long long i = 0; i < nu; ++i) {
      num += std::norm(std::complex<double>(x[i]) - std::complex<double>(w.phantom[i]));
      den += std::norm(std::complex<double>(w.phantom[i]));
    }
    err = std::sqrt(num / den);
  }
  std::printf("{\"imDim\": %d, \"N_u\": [", w.imDim);
  for (int d = 0; d < w.imDim; ++d) std::printf("%s%d", d ? ", " : "", w.N[d]);
  std::printf("], \"n_u\": [");
  for (int d = 0; d < w.imDim; ++d) std::printf("%s%d", d ? ", " : "", w.n[d]);
  std::printf("], \"nPt\": %d, \"nCh\": %d, \"nIter\": %d, \"nCGD\": %d, \"setup_ms\": %.3f, \"recon_ms\": %.3f, "
              "\"residual\": [",
              w.nPt, w.nCh, nIter, nCGD, setup_ms, best_ms);
  for (int i = 0; i < nIter; ++i) std::printf("%s%.17g", i ? ", " : "", res[i]);
  std::printf("]");
  if (err >= 0) std::printf(", \"rel_err_vs_phantom\": %.6f", err);
  std::printf("}\n");
  check(mlg_plan_destroy(plan), "mlg_plan_destroy");
  mlg_matrix_destroy(Gu);
  mlg_matrix_destroy(Gut);
  return 0;
}
