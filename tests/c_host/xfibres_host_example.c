/*
 * A host program that uses libbpx.so through include/bpx.h alone, as the reference's xfibres_gpu
 * host would (CUDA/xfibres_gpu.cc:134-188 calling xfibres_gpu(), CUDA/xfibres_gpu.h:15-23):
 * reads a subpart's data, bvecs and bvals from raw float files, runs bpx_xfibres_host with the
 * options given on the command line and writes the merged samples and means back as raw floats.
 *
 *   xfibres_host_example DIR NVOX NDIR MODEL NFIB NBURN NJUMPS SAMPLEEVERY RICIAN F0 SEED
 *
 * DIR holds data.f32 [nvox][ndir], bvecs.f32 [3][ndir], bvals.f32 [ndir]; the program writes
 * th.f32, ph.f32, f.f32 [nfib][nsamples][nvox] and mean_d.f32, mean_S0.f32 [nvox] there.
 * Exit status 0 on success; errors print bpx_last_error().
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bpx.h"

static float* read_f32(const char* dir, const char* name, size_t n) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  FILE* fp = fopen(path, "rb");
  if (!fp) return NULL;
  float* a = (float*)malloc(n * sizeof(float));
  if (a && fread(a, sizeof(float), n, fp) != n) {
    free(a);
    a = NULL;
  }
  fclose(fp);
  return a;
}

static int write_f32(const char* dir, const char* name, const float* a, size_t n) {
  char path[4096];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  FILE* fp = fopen(path, "wb");
  if (!fp) return 1;
  const int bad = fwrite(a, sizeof(float), n, fp) != n;
  fclose(fp);
  return bad;
}

int main(int argc, char** argv) {
  if (argc != 12) {
    fprintf(stderr, "usage: %s DIR NVOX NDIR MODEL NFIB NBURN NJUMPS SAMPLEEVERY RICIAN F0 SEED\n", argv[0]);
    return 2;
  }
  const char* dir = argv[1];
  const int nvox = atoi(argv[2]), ndir = atoi(argv[3]);
  bpx_options opt;
  bpx_options_default(&opt);
  opt.model = atoi(argv[4]);
  opt.nfibres = atoi(argv[5]);
  opt.nburn = atoi(argv[6]);
  opt.njumps = atoi(argv[7]);
  opt.sampleevery = atoi(argv[8]);
  opt.rician = atoi(argv[9]);
  opt.f0 = atoi(argv[10]);
  opt.seed = (uint64_t)strtoull(argv[11], NULL, 10);
  const int ns = bpx_nsamples(&opt), K = opt.nfibres;
  float* data = read_f32(dir, "data.f32", (size_t)nvox * ndir);
  float* bvecs = read_f32(dir, "bvecs.f32", 3 * (size_t)ndir);
  float* bvals = read_f32(dir, "bvals.f32", (size_t)ndir);
  if (!data || !bvecs || !bvals) {
    fprintf(stderr, "cannot read the inputs in %s\n", dir);
    return 1;
  }
  const size_t nsamp = (size_t)K * ns * nvox;
  float* th = (float*)calloc(nsamp, sizeof(float));
  float* ph = (float*)calloc(nsamp, sizeof(float));
  float* f = (float*)calloc(nsamp, sizeof(float));
  float* md = (float*)calloc(nvox, sizeof(float));
  float* ms0 = (float*)calloc(nvox, sizeof(float));
  bpx_volume vol;
  memset(&vol, 0, sizeof vol);
  vol.nvox = nvox;
  vol.ndir = ndir;
  vol.data = data;
  vol.bvecs = bvecs;
  vol.bvals = bvals;
  bpx_outputs out;
  memset(&out, 0, sizeof out);
  out.th = th;
  out.ph = ph;
  out.f = f;
  out.mean_d = md;
  out.mean_S0 = ms0;
  if (bpx_xfibres_host(&opt, &vol, &out) != BPX_OK) {
    fprintf(stderr, "bpx_xfibres_host: %s\n", bpx_last_error());
    return 1;
  }
  int bad = write_f32(dir, "th.f32", th, nsamp) | write_f32(dir, "ph.f32", ph, nsamp) |
            write_f32(dir, "f.f32", f, nsamp) | write_f32(dir, "mean_d.f32", md, nvox) |
            write_f32(dir, "mean_S0.f32", ms0, nvox);
  free(data);
  free(bvecs);
  free(bvals);
  free(th);
  free(ph);
  free(f);
  free(md);
  free(ms0);
  return bad;
}
