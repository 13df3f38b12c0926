// gso_<steps>.out writer: the per-swarm result files of the reference GPU path
// (source/dock/src/cuda/prepare_gso_task.cu:2838-2905):
//   <dir>/swarm_<i>/gso_<steps>.out, header line, then per glowworm
//   "(p0, p1, ..., p{L-1})\t0\t0\t<luciferin>\t<neighbours>\t<vision range>\t<score>\t\n"
// with every double printed as std::to_string does ("%f").  The reference maps the file with
// O_CREAT and no truncation, so a longer pre-existing file keeps a stale tail; this writer
// truncates.  Also here: the cluster.repr writer and the checkpoint files of a GSO state.
#include <sys/stat.h>
#include <sys/types.h>

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

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

// ---- checkpoints of one complex's GSO state ----
// Layout (native byte order): "SDCKPT01", int32 n_swarms, n_glowworms, pose_len, 0, int64
// steps_done, int64 steps_total, then pos [S][G][pl], scoring, luciferin, vision_range [S][G] (double), step, moved,
// nnei_len, select [S][G] (int32), ligand_reference_pose [S][G][3] (double), and a trailing FNV-1a
// 64-bit hash of everything before it.
namespace {

const char kCkptMagic[8] = {'S', 'D', 'C', 'K', 'P', 'T', '0', '1'};

struct Fnv {
  unsigned long long h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) {
      h ^= b[i];
      h *= 1099511628211ull;
    }
  }
};

struct CkptField {
  void* data;
  size_t bytes;
};

std::vector<CkptField> ckpt_fields(const sd_swarm_state* st, int S, int G, int pl) {
  const size_t n = (size_t)S * G;
  return {{st->pos, n * pl * sizeof(double)},       {st->scoring, n * sizeof(double)},
          {st->luciferin, n * sizeof(double)},      {st->vision_range, n * sizeof(double)},
          {st->step, n * sizeof(int)},              {st->moved, n * sizeof(int)},
          {st->nnei_len, n * sizeof(int)},          {st->select, n * sizeof(int)},
          {st->ligand_reference_pose, n * 3 * sizeof(double)}};
}

bool ckpt_state_complete(const sd_swarm_state* st) {
  return st && st->pos && st->scoring && st->luciferin && st->vision_range && st->step && st->moved &&
         st->nnei_len && st->select && st->ligand_reference_pose;
}

int read_header(std::FILE* f, int dims[4], long long steps[2], Fnv& fnv) {
  char magic[8];
  if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kCkptMagic, 8) != 0) return SD_ERR_ARG;
  if (std::fread(dims, sizeof(int), 4, f) != 4 || std::fread(steps, sizeof(long long), 2, f) != 2) return SD_ERR_ARG;
  fnv.add(magic, 8);
  fnv.add(dims, sizeof(int) * 4);
  fnv.add(steps, sizeof(long long) * 2);
  return SD_OK;
}

}  // namespace

extern "C" int sd_write_checkpoint(const char* path, int n_swarms, int n_glowworms, int pose_len, long long steps_done,
                                   long long steps_total, const sd_swarm_state* st) {
  if (!path || n_swarms <= 0 || n_glowworms <= 0 || pose_len < 7 || steps_done < 0 || steps_total < 0 ||
      !ckpt_state_complete(st))
    return sd::fail(SD_ERR_ARG, "sd_write_checkpoint: bad arguments");
  const std::string tmp = std::string(path) + ".partial";
  std::FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) return sd::fail(SD_ERR_ARG, std::string("sd_write_checkpoint: cannot open ") + tmp);
  Fnv fnv;
  const int dims[4] = {n_swarms, n_glowworms, pose_len, 0};
  const long long steps[2] = {steps_done, steps_total};
  bool ok = std::fwrite(kCkptMagic, 1, 8, f) == 8 && std::fwrite(dims, sizeof(int), 4, f) == 4 &&
            std::fwrite(steps, sizeof(long long), 2, f) == 2;
  fnv.add(kCkptMagic, 8);
  fnv.add(dims, sizeof(dims));
  fnv.add(steps, sizeof(steps));
  for (const CkptField& c : ckpt_fields(st, n_swarms, n_glowworms, pose_len)) {
    ok = ok && std::fwrite(c.data, 1, c.bytes, f) == c.bytes;
    fnv.add(c.data, c.bytes);
  }
  ok = ok && std::fwrite(&fnv.h, sizeof(fnv.h), 1, f) == 1;
  ok = (std::fclose(f) == 0) && ok;
  // the file appears under its name only once complete
  if (!ok || std::rename(tmp.c_str(), path) != 0) {
    std::remove(tmp.c_str());
    return sd::fail(SD_ERR_ARG, std::string("sd_write_checkpoint: cannot write ") + path);
  }
  return SD_OK;
}

extern "C" int sd_checkpoint_info(const char* path, int* n_swarms, int* n_glowworms, int* pose_len,
                                  long long* steps_done, long long* steps_total) {
  if (!path) return sd::fail(SD_ERR_ARG, "sd_checkpoint_info: bad arguments");
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return sd::fail(SD_ERR_ARG, std::string("sd_checkpoint_info: cannot open ") + path);
  int dims[4];
  long long steps[2] = {0, 0};
  Fnv fnv;
  const int rc = read_header(f, dims, steps, fnv);
  std::fclose(f);
  if (rc) return sd::fail(rc, std::string("sd_checkpoint_info: not a checkpoint: ") + path);
  if (n_swarms) *n_swarms = dims[0];
  if (n_glowworms) *n_glowworms = dims[1];
  if (pose_len) *pose_len = dims[2];
  if (steps_done) *steps_done = steps[0];
  if (steps_total) *steps_total = steps[1];
  return SD_OK;
}

extern "C" int sd_read_checkpoint(const char* path, int n_swarms, int n_glowworms, int pose_len, long long* steps_done,
                                  long long* steps_total, sd_swarm_state* st) {
  if (!path || !ckpt_state_complete(st)) return sd::fail(SD_ERR_ARG, "sd_read_checkpoint: bad arguments");
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return sd::fail(SD_ERR_ARG, std::string("sd_read_checkpoint: cannot open ") + path);
  int dims[4];
  long long steps[2] = {0, 0};
  Fnv fnv;
  if (read_header(f, dims, steps, fnv)) {
    std::fclose(f);
    return sd::fail(SD_ERR_ARG, std::string("sd_read_checkpoint: not a checkpoint: ") + path);
  }
  if (dims[0] != n_swarms || dims[1] != n_glowworms || dims[2] != pose_len) {
    std::fclose(f);
    return sd::fail(SD_ERR_ARG, "sd_read_checkpoint: " + std::to_string(dims[0]) + " x " + std::to_string(dims[1]) +
                                    " glowworms of pose length " + std::to_string(dims[2]) +
                                    " in the file, not the sizes asked for");
  }
  bool ok = true;
  for (const CkptField& c : ckpt_fields(st, n_swarms, n_glowworms, pose_len)) {
    ok = ok && std::fread(c.data, 1, c.bytes, f) == c.bytes;
    if (ok) fnv.add(c.data, c.bytes);
  }
  unsigned long long h = 0;
  ok = ok && std::fread(&h, sizeof(h), 1, f) == 1;
  char extra;
  ok = ok && std::fread(&extra, 1, 1, f) == 0;  // nothing after the hash
  std::fclose(f);
  if (!ok || h != fnv.h)
    return sd::fail(SD_ERR_ARG, std::string("sd_read_checkpoint: truncated or corrupted: ") + path);
  if (steps_done) *steps_done = steps[0];
  if (steps_total) *steps_total = steps[1];
  return SD_OK;
}
