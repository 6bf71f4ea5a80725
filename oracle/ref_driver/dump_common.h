// Shared helpers for the reference dump drivers (test infrastructure only).
//
// The drivers link the compiled reference (oracle/_ref) and write raw
// little-endian arrays into an output directory: one file per array, named
// "<tag>.<type>" with type in {i32, f64}, plus a "meta.txt" of key=value lines.
// The Python side (oracle/refdump.py) reads them back with numpy.fromfile.
#ifndef CDGPU_DUMP_COMMON_H
#define CDGPU_DUMP_COMMON_H

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

static std::string g_outdir;
static FILE *g_meta = nullptr;

static void dump_open(const char *dir)
{
  g_outdir = dir ? dir : "";
  if (g_outdir.empty()) return;
  std::string m = g_outdir + "/meta.txt";
  g_meta = fopen(m.c_str(), "w");
  if (!g_meta) { fprintf(stderr, "cannot open %s\n", m.c_str()); exit(2); }
}

static void dump_i32(const std::string &tag, const int *p, long n)
{
  if (g_outdir.empty()) return;
  std::string fn = g_outdir + "/" + tag + ".i32";
  FILE *f = fopen(fn.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot open %s\n", fn.c_str()); exit(2); }
  if (n > 0) fwrite(p, sizeof(int), n, f);
  fclose(f);
}

static void dump_f64(const std::string &tag, const double *p, long n)
{
  if (g_outdir.empty()) return;
  std::string fn = g_outdir + "/" + tag + ".f64";
  FILE *f = fopen(fn.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot open %s\n", fn.c_str()); exit(2); }
  if (n > 0) fwrite(p, sizeof(double), n, f);
  fclose(f);
}

static void meta_i(const std::string &key, long v)
{
  if (g_meta) { fprintf(g_meta, "%s=%ld\n", key.c_str(), v); fflush(g_meta); }
}

static void meta_d(const std::string &key, double v)
{
  if (g_meta) { fprintf(g_meta, "%s=%.17g\n", key.c_str(), v); fflush(g_meta); }
}

static double wall_now()
{
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

static std::string lvl(int l, const char *name)
{
  return "L" + std::to_string(l) + "_" + name;
}

#endif
