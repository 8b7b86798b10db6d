// Kernel-only timing of the reference's geo2rdr and crossmul kernels on
// device-resident inputs.  Test infrastructure: the reference arm of the
// benchmark runs it beside the reference executables, so that the
// reference's own kernels (deramp_burst, reproject and
// find_first_last_nonzero_rows_kernel of csrc/src/geo2rdr.cu:86-299;
// conj_mul, cpx_col_look and cpx_row_look of csrc/src/sario.cu:199-286, as
// crossmul_daemon.cu:921-975 launches them) are timed without process
// start-up, SQLite or file I/O.
//
// The reference source is compiled where it lies: this file includes
// csrc/src/geo2rdr.cu (its main renamed) and is linked with the other
// sources of the geo2rdr executable.  Launch configurations are the
// reference's (256-thread blocks, one thread per element).
//
// Usage: kbench_chain <manifest> <reps> <ifg_out>
//   manifest: "key value" lines (scalars and paths of raw arrays) for the
//   two bursts of a pair ("ref_*", "sec_*") and the crossmul box; written by
//   the benchmark from the oracle's restatement of the host computations.
// Prints one JSON line of per-kernel times (ms, median over reps after one
// warm-up) and writes the looked interferogram (complex64) to ifg_out.
#define main ref_geo2rdr_main
#include "geo2rdr.cu"
#undef main

#include <algorithm>
#include <map>
#include <vector>

namespace kb {

struct Manifest {
  std::map<std::string, std::string> kv;
  explicit Manifest(const std::string &path) {
    std::ifstream f(path);
    std::string k, v;
    while (f >> k >> v) kv[k] = v;
  }
  const std::string &str(const std::string &k) const {
    auto it = kv.find(k);
    if (it == kv.end()) {
      std::cerr << "kbench_chain: manifest lacks " << k << std::endl;
      std::exit(2);
    }
    return it->second;
  }
  double num(const std::string &k) const { return std::stod(str(k)); }
  int integer(const std::string &k) const { return std::stoi(str(k)); }
};

template <typename T>
std::vector<T> load(const std::string &path, size_t n) {
  std::vector<T> v(n);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char *>(v.data()), sizeof(T) * n);
  if (!f) {
    std::cerr << "kbench_chain: short read of " << path << std::endl;
    std::exit(2);
  }
  return v;
}

template <typename T>
T *upload(const std::vector<T> &h) {
  T *d = nullptr;
  CHECK_CUDA(cudaMalloc((void **)&d, sizeof(T) * std::max<size_t>(h.size(), 1)));
  CHECK_CUDA(cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return d;
}

struct Burst {
  int L, S, nstat, nrow, ncol, win_left, win_top, fvl, lvl, fvs, lvs;
  double tmid, latmax0, lonmin0, dlat, dlon, rngstart, tstart, dmrg, dtaz, etac0, ks, wvl;
  double fm[4], dc[4], xmid[3], vmid[3];
  Complex *d_slc0, *d_burst, *d_out;
  double *d_kt, *d_eta, *d_etaref, *d_tt, *d_xx, *d_vv, *d_xmid, *d_vmid;
  short int *d_dem;
  int *d_first, *d_last;
  int first = 0, last = 0;

  Burst(const Manifest &m, const std::string &p) {
    L = m.integer(p + "L");
    S = m.integer(p + "S");
    nstat = m.integer(p + "nstat");
    nrow = m.integer(p + "nrow");
    ncol = m.integer(p + "ncol");
    win_left = m.integer(p + "win_left");
    win_top = m.integer(p + "win_top");
    fvl = m.integer(p + "fvl");
    lvl = m.integer(p + "lvl");
    fvs = m.integer(p + "fvs");
    lvs = m.integer(p + "lvs");
    tmid = m.num(p + "tmid");
    latmax0 = m.num(p + "latmax0");
    lonmin0 = m.num(p + "lonmin0");
    dlat = m.num(p + "dlat");
    dlon = m.num(p + "dlon");
    rngstart = m.num(p + "rngstart");
    tstart = m.num(p + "tstart");
    dmrg = m.num(p + "dmrg");
    dtaz = m.num(p + "dtaz");
    etac0 = m.num(p + "etac0");
    ks = m.num(p + "ks");
    wvl = m.num(p + "wvl");
    for (int i = 0; i < 4; ++i) {
      fm[i] = m.num(p + "fm" + std::to_string(i));
      dc[i] = m.num(p + "dc" + std::to_string(i));
    }
    for (int i = 0; i < 3; ++i) {
      xmid[i] = m.num(p + "xmid" + std::to_string(i));
      vmid[i] = m.num(p + "vmid" + std::to_string(i));
    }
    d_slc0 = upload(load<Complex>(m.str(p + "slc"), (size_t)L * S));
    CHECK_CUDA(cudaMalloc((void **)&d_burst, sizeof(Complex) * (size_t)L * S));
    CHECK_CUDA(cudaMalloc((void **)&d_out, sizeof(Complex) * (size_t)nrow * ncol));
    d_kt = upload(load<double>(m.str(p + "kt"), S));
    d_etaref = upload(load<double>(m.str(p + "etaref"), S));
    d_eta = upload(load<double>(m.str(p + "eta"), L));
    d_tt = upload(load<double>(m.str(p + "tt"), nstat));
    d_xx = upload(load<double>(m.str(p + "xx"), 3 * (size_t)nstat));
    d_vv = upload(load<double>(m.str(p + "vv"), 3 * (size_t)nstat));
    d_xmid = upload(std::vector<double>(xmid, xmid + 3));
    d_vmid = upload(std::vector<double>(vmid, vmid + 3));
    d_dem = upload(load<short int>(m.str(p + "dem"), (size_t)nrow * ncol));
    CHECK_CUDA(cudaMalloc((void **)&d_first, sizeof(int)));
    CHECK_CUDA(cudaMalloc((void **)&d_last, sizeof(int)));
  }
};

float median(std::vector<float> v) {
  std::sort(v.begin(), v.end());
  return v.empty() ? 0.f : v[v.size() / 2];
}

}  // namespace kb

int main(int argc, char *argv[]) {
  if (argc < 4) {
    std::cerr << "usage: kbench_chain <manifest> <reps> <ifg_out>" << std::endl;
    return 2;
  }
  kb::Manifest m(argv[1]);
  const int reps = std::max(1, std::atoi(argv[2]));
  kb::Burst b[2] = {kb::Burst(m, "ref_"), kb::Burst(m, "sec_")};
  const int blockSize = 256;
  cudaEvent_t e[4];
  for (auto &x : e) CHECK_CUDA(cudaEventCreate(&x));
  std::vector<float> t_der[2], t_rep[2], t_rows[2], t_xm;
  // crossmul box in RSC coordinates, aligned to the looks by crossmul_daemon
  const int bl = m.integer("box_left"), bt = m.integer("box_top"), br = m.integer("box_right"),
            bb = m.integer("box_bottom"), rl = m.integer("rowlook"), cl = m.integer("collook");
  const int nrow_b = bb - bt, ncol_b = br - bl, nrow_sm = nrow_b / rl, ncol_sm = ncol_b / cl;
  for (const kb::Burst &x : b)  // the box must lie inside both geocoded windows
    if (nrow_b <= 0 || ncol_b <= 0 || rl < 1 || cl < 1 || bl < x.win_left || bt < x.win_top ||
        br > x.win_left + x.ncol || bb > x.win_top + x.nrow) {
      std::cerr << "kbench_chain: crossmul box outside a window" << std::endl;
      return 2;
    }
  Complex *d_c[2], *d_ifg, *d_ifgc, *d_ifgl;
  for (auto &p : d_c) CHECK_CUDA(cudaMalloc((void **)&p, sizeof(Complex) * (size_t)nrow_b * ncol_b));
  CHECK_CUDA(cudaMalloc((void **)&d_ifg, sizeof(Complex) * (size_t)nrow_b * ncol_b));
  CHECK_CUDA(cudaMalloc((void **)&d_ifgc, sizeof(Complex) * (size_t)nrow_b * ncol_sm));
  CHECK_CUDA(cudaMalloc((void **)&d_ifgl, sizeof(Complex) * (size_t)nrow_sm * ncol_sm));
  for (int rep = 0; rep <= reps; ++rep) {
    for (int q = 0; q < 2; ++q) {
      kb::Burst &x = b[q];
      const size_t burstsize = (size_t)x.L * x.S;
      CHECK_CUDA(cudaMemcpy(x.d_burst, x.d_slc0, sizeof(Complex) * burstsize, cudaMemcpyDeviceToDevice));
      int h_first = x.nrow, h_last = -1;
      CHECK_CUDA(cudaMemcpy(x.d_first, &h_first, sizeof(int), cudaMemcpyHostToDevice));
      CHECK_CUDA(cudaMemcpy(x.d_last, &h_last, sizeof(int), cudaMemcpyHostToDevice));
      CHECK_CUDA(cudaDeviceSynchronize());
      const int numBlocks = (int)((burstsize + blockSize - 1) / blockSize);
      cudaEventRecord(e[0]);
      deramp_burst<<<numBlocks, blockSize>>>(x.d_kt, x.d_eta, x.d_etaref, x.d_burst, x.S, burstsize);
      cudaEventRecord(e[1]);
      const int demBlocks = (x.nrow * x.ncol + blockSize - 1) / blockSize;
      reproject<<<demBlocks, blockSize>>>(x.d_dem, x.d_burst, x.d_out, x.d_tt, x.d_xx, x.d_vv, x.nstat, x.tmid,
                                          x.d_xmid, x.d_vmid, x.latmax0, x.lonmin0, x.dlat, x.dlon, x.ncol,
                                          x.rngstart, x.tstart, x.dmrg, x.dtaz, x.S, x.L, x.fm[0], x.fm[1], x.fm[2],
                                          x.fm[3], x.dc[0], x.dc[1], x.dc[2], x.dc[3], x.etac0, x.ks, x.fvl, x.lvl,
                                          x.fvs, x.lvs, x.wvl, (size_t)x.nrow * x.ncol);
      cudaEventRecord(e[2]);
      find_nonzero_rows(x.d_out, x.nrow, x.ncol, x.d_first, x.d_last, x.first, x.last);
      cudaEventRecord(e[3]);
      CHECK_CUDA(cudaEventSynchronize(e[3]));
      CHECK_CUDA(cudaGetLastError());
      float a, c, d;
      cudaEventElapsedTime(&a, e[0], e[1]);
      cudaEventElapsedTime(&c, e[1], e[2]);
      cudaEventElapsedTime(&d, e[2], e[3]);
      if (rep > 0) {
        t_der[q].push_back(a);
        t_rep[q].push_back(c);
        t_rows[q].push_back(d);
      }
      // the daemon's crop of the box out of the geocoded window (host side in
      // the daemon, untimed here)
      CHECK_CUDA(cudaMemcpy2D(d_c[q], sizeof(Complex) * ncol_b,
                              x.d_out + (size_t)(bt - x.win_top) * x.ncol + (bl - x.win_left),
                              sizeof(Complex) * x.ncol, sizeof(Complex) * ncol_b, nrow_b,
                              cudaMemcpyDeviceToDevice));
    }
    CHECK_CUDA(cudaDeviceSynchronize());
    cudaEventRecord(e[0]);
    conj_mul<<<(int)(((size_t)nrow_b * ncol_b + blockSize - 1) / blockSize), blockSize>>>(d_c[0], d_c[1], d_ifg,
                                                                                          (size_t)nrow_b * ncol_b);
    Complex *cur = d_ifg;
    if (cl > 1) {
      cpx_col_look<<<(int)(((size_t)nrow_b * ncol_sm + blockSize - 1) / blockSize), blockSize>>>(
          d_ifg, d_ifgc, cl, ncol_b, (size_t)nrow_b * ncol_sm);
      cur = d_ifgc;
    }
    if (rl > 1) {
      cpx_row_look<<<(int)(((size_t)nrow_sm * ncol_sm + blockSize - 1) / blockSize), blockSize>>>(
          cur, d_ifgl, rl, ncol_sm, (size_t)nrow_sm * ncol_sm);
      cur = d_ifgl;
    }
    cudaEventRecord(e[1]);
    CHECK_CUDA(cudaEventSynchronize(e[1]));
    CHECK_CUDA(cudaGetLastError());
    float a;
    cudaEventElapsedTime(&a, e[0], e[1]);
    if (rep > 0) t_xm.push_back(a);
    if (rep == reps) {
      std::vector<Complex> h((size_t)nrow_sm * ncol_sm);
      CHECK_CUDA(cudaMemcpy(h.data(), cur, sizeof(Complex) * h.size(), cudaMemcpyDeviceToHost));
      std::ofstream f(argv[3], std::ios::binary);
      f.write(reinterpret_cast<const char *>(h.data()), sizeof(Complex) * h.size());
    }
  }
  std::printf("{\"deramp_ms\": [%.6f, %.6f], \"reproject_ms\": [%.6f, %.6f], \"nonzero_rows_ms\": [%.6f, %.6f], "
              "\"crossmul_looks_ms\": %.6f, \"burst_px\": [%d, %d], \"geo_px\": [%d, %d], "
              "\"crop_rows\": [[%d, %d], [%d, %d]], \"ifg_shape\": [%d, %d], \"reps\": %d}\n",
              kb::median(t_der[0]), kb::median(t_der[1]), kb::median(t_rep[0]), kb::median(t_rep[1]),
              kb::median(t_rows[0]), kb::median(t_rows[1]), kb::median(t_xm), b[0].L * b[0].S, b[1].L * b[1].S,
              b[0].nrow * b[0].ncol, b[1].nrow * b[1].ncol, b[0].first, b[0].last, b[1].first, b[1].last, nrow_sm,
              ncol_sm, reps);
  return 0;
}
