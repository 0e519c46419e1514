// sgt_cli.cpp -- drop-in for the reference's command line tools
//   sg_tsne_cuda     (CU/testing_modules/demo_perplexity.cu:32-213)
//   demo_stochastic_matrix (CU/testing_modules/demo_stochastic_matrix.cu)
//
// Usage: sg_tsne_cuda [-d D] [-a alpha] [-m max_iter] [-e early_iter] [-h h]
//                     [-p np] [-u perplexity] [-f err] [-g ng] [-s sim]
//                     [-n points] [-t coo|hybrid|csr|2|3|0] [-l lambda]
//                     [-G fixed|h] [-k kNN-file-is-P: 0|1] [-b 0|1] FILE
// FILE holds either a sparse stochastic matrix in Matrix Market coordinate
// format (1-based "row col value", as buildPFromMTX, CU/utils.cu:335-409) or
// dense points ("n d" then n*d values, as readXfromMTX, CU/utils.cu:216-256;
// -n takes the first n points).  Dense input goes through the stages of the
// reference's demo_perplexity.cu:111-158 on the device: exact kNN with
// ceil(3u) neighbours (sgt_knn, where the reference calls FLANN), distances
// divided by their maximum, perplexity equalisation to u (sgt_perplexity),
// then sgt_embed.
// Initial coordinates come from yin2m.txt in the working directory when it
// exists (as the reference's demo), else 1e-4 N(0,1).
// Outputs: sgtsneEmbedding.txt (one point per line, as extractEmbeddingTextT)
// and timeInfo.txt (appended, as ExtractTimeInfo); with -b 1 also
// embedding.bin, the n*d FP32 coordinates dimension-major as the reference's
// sgtsneCUDA returns them, written raw as extractEmbedding (CU/utils.cu:140-148).
#include "sgtsne_b200.h"

#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>


static int parse_format(const char *s) {
  if (!strcmp(s, "coo") || !strcmp(s, "2")) return SGT_FORMAT_COO;
  if (!strcmp(s, "hybrid") || !strcmp(s, "3")) return SGT_FORMAT_HYBRID;
  if (!strcmp(s, "csr") || !strcmp(s, "0")) return SGT_FORMAT_CSR;
  return -1;
}

static bool read_mtx(const std::string &fn, int &n, std::vector<int> &rp, std::vector<int> &col,
                     std::vector<float> &val) {
  std::ifstream fin(fn);
  if (!fin) return false;
  std::string line;
  bool header = false;
  while (fin.peek() == '%') {
    std::getline(fin, line);
    header = true;
  }
  (void)header;
  long m, nn, nnz;
  if (!(fin >> m >> nn >> nnz)) return false;
  n = (int)m;
  std::vector<int> r(nnz), c(nnz);
  std::vector<float> v(nnz);
  for (long l = 0; l < nnz; l++)
    if (!(fin >> r[l] >> c[l] >> v[l])) return false;
  // column-major input (CSC of the reference) read as rows of P^T: the
  // reference treats P as column-stochastic; store row = column index.
  rp.assign(n + 1, 0);
  for (long l = 0; l < nnz; l++) rp[c[l]]++;
  for (int i = 0; i < n; i++) rp[i + 1] += rp[i];
  col.resize(nnz);
  val.resize(nnz);
  std::vector<int> fill(rp.begin(), rp.end() - 1);
  for (long l = 0; l < nnz; l++) {
    const int cc = c[l] - 1;
    col[fill[cc]] = r[l] - 1;
    val[fill[cc]] = v[l];
    fill[cc]++;
  }
  return true;
}

static bool read_dense(const std::string &fn, int limit, int &n, int &dim,
                       std::vector<float> &X) {
  std::ifstream fin(fn);
  if (!fin) return false;
  long nn, dd;
  if (!(fin >> nn >> dd) || nn < 2 || dd < 1) return false;
  if (limit > 0 && limit < nn) nn = limit;
  n = (int)nn;
  dim = (int)dd;
  X.resize((size_t)n * dim);
  for (size_t l = 0; l < X.size(); l++)
    if (!(fin >> X[l])) return false;
  return true;
}

// kNN -> max-normalised distances -> perplexity rows, as host CSR with
// ceil(3u) entries per row (CU/testing_modules/demo_perplexity.cu:98-158)
static sgt_status dense_to_p(sgt_ctx *ctx, int n, int dim, const std::vector<float> &X, float u,
                             std::vector<int> &rp, std::vector<int> &col,
                             std::vector<float> &val) {
  const int nn = (int)std::ceil(u * 3);
  if (nn >= n) return SGT_ERR_INVALID_ARG;
  float *dX = nullptr, *dD = nullptr, *dP = nullptr;
  int *dI = nullptr;
  const size_t m = (size_t)n * nn;
  sgt_status st = SGT_OK;
  if (cudaMalloc(&dX, sizeof(float) * X.size()) != cudaSuccess ||
      cudaMalloc(&dD, sizeof(float) * m) != cudaSuccess ||
      cudaMalloc(&dP, sizeof(float) * m) != cudaSuccess ||
      cudaMalloc(&dI, sizeof(int) * m) != cudaSuccess)
    st = SGT_ERR_NO_MEMORY;
  if (st == SGT_OK &&
      cudaMemcpy(dX, X.data(), sizeof(float) * X.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    st = SGT_ERR_CUDA;
  if (st == SGT_OK) st = sgt_knn(ctx, n, dim, dX, nn, dI, dD);
  std::vector<float> D(m);
  if (st == SGT_OK &&
      cudaMemcpy(D.data(), dD, sizeof(float) * m, cudaMemcpyDeviceToHost) != cudaSuccess)
    st = SGT_ERR_CUDA;
  if (st == SGT_OK) {
    float mx = 0.f;
    for (float v : D) mx = std::max(mx, v);
    if (mx > 0)
      for (float &v : D) v /= mx;
    if (cudaMemcpy(dD, D.data(), sizeof(float) * m, cudaMemcpyHostToDevice) != cudaSuccess)
      st = SGT_ERR_CUDA;
  }
  if (st == SGT_OK) st = sgt_perplexity(ctx, n, nn, dD, u, dP, nullptr);
  if (st == SGT_OK) {
    col.resize(m);
    val.resize(m);
    rp.resize((size_t)n + 1);
    for (int i = 0; i <= n; i++) rp[i] = i * nn;
    if (cudaMemcpy(col.data(), dI, sizeof(int) * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(val.data(), dP, sizeof(float) * m, cudaMemcpyDeviceToHost) != cudaSuccess)
      st = SGT_ERR_CUDA;
  }
  cudaFree(dX);
  cudaFree(dD);
  cudaFree(dP);
  cudaFree(dI);
  return st;
}

int main(int argc, char **argv) {
  if (argc <= 1 || argv[argc - 1][0] == '-') {
    std::cerr << "No filename provided!" << std::endl;
    return 1;
  }
  std::string filename = argv[argc - 1];
  sgt_params p;
  sgt_params_default(&p);
  float u = 30;
  int mtx_mode = -1, write_bin = 0;
  opterr = 0;
  int opt;
  while ((opt = getopt(argc, argv, "d:a:m:e:h:p:u:f:g:s:n:t:l:G:k:b:")) != -1) {
    switch (opt) {
      case 'd': p.d = atoi(optarg); break;
      case 'm': p.max_iter = atoi(optarg); break;
      case 'e': p.early_iter = atoi(optarg); break;
      case 'p': p.np = atoi(optarg); break;
      case 'u': u = (float)atof(optarg); break;
      case 'a': p.alpha = (float)atof(optarg); break;
      case 'h': p.h = (float)atof(optarg); break;
      case 'f': p.compute_error = atoi(optarg); break;
      case 'g': p.ng = atoi(optarg); break;
      case 's': p.sim = atoi(optarg); break;
      case 'n': p.n = atoi(optarg); break;
      case 'l': p.lambda = (float)atof(optarg); break;
      case 't': {
        const int f = parse_format(optarg);
        if (f < 0) {
          std::cerr << "Unknown format: " << optarg << std::endl;
          return 1;
        }
        p.format = f;
        break;
      }
      case 'G': p.grid_mode = !strcmp(optarg, "fixed") ? SGT_GRID_FIXED : SGT_GRID_H; break;
      case 'k': mtx_mode = atoi(optarg); break;
      case 'b': write_bin = atoi(optarg); break;
      case '?': std::cerr << "Unknown option: '" << char(optopt) << "'!" << std::endl; break;
    }
  }
  sgt_ctx *ctx = nullptr;
  sgt_status st = sgt_create(0, &ctx);
  if (st != SGT_OK) {
    std::cerr << "sgt_create: " << sgt_status_string(st) << std::endl;
    return 2;
  }
  int n = 0;
  std::vector<int> rp, col;
  std::vector<float> val;
  // decide the input kind from the first line: "%" or three numbers = MTX
  {
    std::ifstream fin(filename);
    if (!fin) {
      std::cerr << "cannot open " << filename << std::endl;
      return 1;
    }
    std::string first;
    std::getline(fin, first);
    if (mtx_mode < 0) {
      std::istringstream is(first);
      double a, b, c;
      mtx_mode = (first.size() && first[0] == '%') || (bool)(is >> a >> b >> c);
    }
  }
  if (mtx_mode) {
    if (!read_mtx(filename, n, rp, col, val)) {
      std::cerr << "cannot parse matrix " << filename << std::endl;
      return 1;
    }
  } else {
    int dim = 0;
    std::vector<float> X;
    if (!read_dense(filename, p.n, n, dim, X)) {
      std::cerr << "cannot parse points " << filename << std::endl;
      sgt_destroy(ctx);
      return 1;
    }
    std::cout << "Number of points " << n << " dimensions " << dim << std::endl;
    st = dense_to_p(ctx, n, dim, X, u, rp, col, val);
    if (st != SGT_OK) {
      std::cerr << "kNN / perplexity: " << sgt_status_string(st) << ": " << sgt_last_error(ctx)
                << std::endl;
      sgt_destroy(ctx);
      return 2;
    }
  }
  p.n = n;
  std::vector<float> y((size_t)n * (p.d > 0 ? p.d : 2));
  std::vector<double> timeinfo(7003, 0.0);
  // initial coordinates from yin2m.txt when it exists (one point per line,
  // stored dim-major), as demo_perplexity.cu:175-185; random otherwise
  std::vector<float> yin;
  {
    std::ifstream yinf("yin2m.txt");
    if (yinf) {
      yin.resize((size_t)n * p.d);
      bool ok = true;
      for (int i = 0; i < n && ok; i++)
        for (int j = 0; j < p.d && ok; j++) ok = (bool)(yinf >> yin[i + (size_t)j * n]);
      if (!ok) {
        std::cerr << "yin2m.txt holds fewer than n*d values; using random Y0" << std::endl;
        yin.clear();
      }
    }
  }
  const auto t0 = std::chrono::steady_clock::now();
  st = sgt_embed(ctx, n, rp.data(), col.data(), val.data(), &p, yin.empty() ? nullptr : yin.data(),
                 y.data(), timeinfo.data());
  timeinfo[7002] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (st != SGT_OK) {
    std::cerr << "sgt_embed: " << sgt_status_string(st) << ": " << sgt_last_error(ctx) << std::endl;
    sgt_destroy(ctx);
    return 2;
  }
  {
    std::ofstream f("sgtsneEmbedding.txt");
    for (int i = 0; i < n; i++) {
      for (int j = 0; j < p.d; j++) f << y[i + (size_t)j * n] << " ";
      f << "\n";
    }
  }
  if (write_bin) {
    FILE *fb = fopen("embedding.bin", "wb");
    if (!fb || fwrite(y.data(), sizeof(float), (size_t)n * p.d, fb) != (size_t)n * p.d) {
      std::cerr << "cannot write embedding.bin" << std::endl;
      if (fb) fclose(fb);
      sgt_destroy(ctx);
      return 3;
    }
    fclose(fb);
  }
  {
    // appended in the layout of ExtractTimeInfo (CU/utils.cu:72-92); the
    // reference writes only when the file already exists, this tool always
    std::ofstream f("timeInfo.txt", std::ios::app);
    f << "N d gds matrix total: \n";
    f << n << " " << p.d << " " << timeinfo[7000] << " " << timeinfo[7001] << " "
      << timeinfo[7002] << "\n";
    f << "Fattr S2G G2G G2S Phi2F Nuconv Pre";
    for (int i = 0; i < 1000; i++) {
      for (int j = 0; j < 7; j++) f << timeinfo[i * 7 + j] << " ";
      f << "\n";
    }
  }
  printf("Total time=%lf\n", timeinfo[7002]);
  sgt_destroy(ctx);
  return 0;
}
