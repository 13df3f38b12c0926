// gso_<steps>.out writer: the per-swarm result files of the reference GPU path
// (source/dock/src/cuda/prepare_gso_task.cu:2838-2905):
//   <dir>/swarm_<i>/gso_<steps>.out, header line, then per glowworm
//   "(p0, p1, ..., p{L-1})\t0\t0\t<luciferin>\t<neighbours>\t<vision range>\t<score>\t\n"
// with every double printed as std::to_string does ("%f").  The reference maps the file with
// O_CREAT and no truncation, so a longer pre-existing file keeps a stale tail; this writer
// truncates.
#include <sys/stat.h>
#include <sys/types.h>

#include <cerrno>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>

#include "sd_internal.h"

extern "C" int sd_write_gso_output(const char* dir, int swarm_offset, int n_swarms, int n_glowworms, int pose_len,
                                   int steps, const double* pos, const double* luciferin, const int* nnei_len,
                                   const double* vision_range, const double* scoring) {
  if (!dir || n_swarms <= 0 || n_glowworms <= 0 || pose_len <= 0 || !pos || !luciferin || !nnei_len ||
      !vision_range || !scoring || swarm_offset < 0)
    return sd::fail(SD_ERR_ARG, "sd_write_gso_output: bad arguments");
  std::string line;
  char num[64];
  for (int s = 0; s < n_swarms; ++s) {
    const std::string sdir = std::string(dir) + "/swarm_" + std::to_string(s + swarm_offset);
    if (mkdir(sdir.c_str(), 0777) != 0 && errno != EEXIST)
      return sd::fail(SD_ERR_ARG, "sd_write_gso_output: cannot create " + sdir);
    const std::string path = sdir + "/gso_" + std::to_string(steps) + ".out";
    FILE* f = fopen(path.c_str(), "w");
    if (!f) return sd::fail(SD_ERR_ARG, "sd_write_gso_output: cannot open " + path);
    std::string buf = "#Coordinates  RecID  LigID  Luciferin  Neighbor's number  Vision Range  Scoring\n";
    for (int g = 0; g < n_glowworms; ++g) {
      const size_t k = (size_t)s * n_glowworms + g;
      line = "(";
      for (int p = 0; p < pose_len; ++p) {
        snprintf(num, sizeof num, "%f", pos[k * pose_len + p]);
        line += num;
        if (p < pose_len - 1) line += ", ";
      }
      line += ")\t0\t0\t";
      snprintf(num, sizeof num, "%f", luciferin[k]);
      line += num;
      line += "\t" + std::to_string(nnei_len[k]) + "\t";
      snprintf(num, sizeof num, "%f", vision_range[k]);
      line += num;
      line += "\t";
      snprintf(num, sizeof num, "%f", scoring[k]);
      line += num;
      line += "\t\n";
      buf += line;
    }
    const bool ok = fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    if (fclose(f) != 0 || !ok) return sd::fail(SD_ERR_ARG, "sd_write_gso_output: write failed for " + path);
  }
  return SD_OK;
}

// cluster.repr (source/dock/src/cuda/pipeline:2936-2944): per cluster of a swarm
//   "<c>:<size>:<score of the representative>:<representative>:lightdock_<representative>.pdb"
// with the score printed by an ostream at its default precision.  The reference reads the score
// at the representative's index of the first swarm for every swarm; this writer takes the
// representative's own swarm.
extern "C" int sd_write_cluster_repr(const char* dir, int swarm_offset, int n_swarms, int n_glowworms,
                                     const int* n_clusters, const int* cluster_rep, const int* cluster_len,
                                     const double* scoring) {
  if (!dir || n_swarms <= 0 || n_glowworms <= 0 || !n_clusters || !cluster_rep || !cluster_len || !scoring ||
      swarm_offset < 0)
    return sd::fail(SD_ERR_ARG, "sd_write_cluster_repr: bad arguments");
  for (int s = 0; s < n_swarms; ++s) {
    const std::string sdir = std::string(dir) + "/swarm_" + std::to_string(s + swarm_offset);
    if (mkdir(sdir.c_str(), 0777) != 0 && errno != EEXIST)
      return sd::fail(SD_ERR_ARG, "sd_write_cluster_repr: cannot create " + sdir);
    std::ostringstream os;
    const size_t b = (size_t)s * n_glowworms;
    if (n_clusters[s] < 0 || n_clusters[s] > n_glowworms)
      return sd::fail(SD_ERR_ARG, "sd_write_cluster_repr: bad cluster count");
    for (int c = 0; c < n_clusters[s]; ++c) {
      const int id = cluster_rep[b + c];
      if (id < 0 || id >= n_glowworms) return sd::fail(SD_ERR_ARG, "sd_write_cluster_repr: bad representative");
      os << c << ":" << cluster_len[b + c] << ":" << scoring[b + id] << ":" << id << ":lightdock_" << id << ".pdb\n";
    }
    std::ofstream f(sdir + "/cluster.repr", std::ios::trunc);
    if (!f) return sd::fail(SD_ERR_ARG, "sd_write_cluster_repr: cannot write " + sdir + "/cluster.repr");
    f << os.str();
  }
  return SD_OK;
}
