// lightdock_b200: the reference's command line (source/simulation/run_simulation.cc:21-129,
// `lightdock -f setup.json -s STEPS -l N`) over the C ABI.
//
// setup.json keys read as in get_setup (source/prep/src/read_input_structure.cc:6-59):
//   swarms, glowworms, anm_rec, anm_lig, use_anm, starting_points_seed, and the GSO keys
//   rho, gamma, beta, initialLuciferin, initialVisionRange, maximumVisionRange,
//   maximumNeighbors (read but unused by the reference; honoured here, reference defaults when
//   absent).  Keys added by this build:
//   "scoring": "dfire" | "pydock"                (absent: dfire)
//   "precision": "mixed" | "fp64" | "fp64_ref"  (absent: mixed)
//   "translation_step", "rotation_step", "nmodes_step"   (absent: the reference's 0.5)
//   receptor_pdb, ligand_pdb, noxt, noh, now: the structures, read as the reference's setup
//        reads them (sd_structure_load); with use_anm, normal modes from sd_anm (cal_anm, which
//        also re-centres each structure on its mean) with anm_rec_rmsd / anm_lig_rmsd (absent:
//        0.5, lightdock's default); swarm centres and starting poses from sd_place_swarms (the
//        reference's surface-based placement) with starting_points_seed, anm_seed (absent:
//        324324) and swarm_radius (absent: 10); membrane, transmembrane and dense_sampling are
//        refused (the reference leaves them undeveloped); pyDock charges are seeded stand-ins
//   "synthetic": {"receptor_atoms": N, "ligand_atoms": M, "seed": s}
//        seeded synthetic receptor/ligand in place of receptor_pdb / ligand_pdb
//   "checkpoint_every": N   write <dir>/checkpoint.ckpt (sd_write_checkpoint) every N steps and
//        at the end.  -t STOP runs only the first STOP of the -s steps and writes the checkpoint
//        (a segment of the run; no result files); -r CHECKPOINT resumes from a checkpoint of the
//        same setup.json and -s (the reference's draws depend on -s: other values are refused)
//   "dfire_table": path of a DCparams-format file (168*168*20 values, one per line);
//        absent: seeded synthetic table ("table_seed", default 3)
// -s STEPS is honoured (the reference parses it but runs its compiled STEPS macro).
// <dir>/run.json: the run's counts, timings, the scorer's rare-path counters and, for mixed
// precision, the autotuned kernel variant.
// Output: <dir>/swarm_<i>/gso_<STEPS>.out as the reference GPU path writes them; with PDB inputs
// also <dir>/swarm_<i>/cluster.repr (sd_cluster on the CA / P atoms) and the final poses as
// <dir>/swarm_<i>/lightdock_<g>.pdb (sd_materialise_poses + sd_write_pose_pdb, the reference
// pipeline's format), per "write_poses": "representatives" (absent: the glowworms cluster.repr
// names), "all" (every glowworm, as the reference's pipeline writes them) or "none".
#include <errno.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sparkle_b200.h"

namespace {

// ---- minimal JSON reader (objects, arrays, strings, numbers, true/false/null) ----
struct JVal {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
  bool b = false;
  double num = 0;
  std::string str;
  std::vector<JVal> arr;
  std::map<std::string, JVal> obj;
  const JVal* get(const std::string& k) const {
    auto it = obj.find(k);
    return it == obj.end() ? nullptr : &it->second;
  }
};

struct JParser {
  const std::string& s;
  size_t i = 0;
  std::string err;
  explicit JParser(const std::string& t) : s(t) {}
  void ws() {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\n' || s[i] == '\t' || s[i] == '\r')) ++i;
  }
  bool fail(const std::string& m) {
    if (err.empty()) err = m + " at offset " + std::to_string(i);
    return false;
  }
  bool value(JVal& v) {
    ws();
    if (i >= s.size()) return fail("unexpected end of input");
    const char c = s[i];
    if (c == '{') return object(v);
    if (c == '[') return array(v);
    if (c == '"') {
      v.kind = JVal::Str;
      return string(v.str);
    }
    if (!s.compare(i, 4, "true")) {
      v.kind = JVal::Bool;
      v.b = true;
      i += 4;
      return true;
    }
    if (!s.compare(i, 5, "false")) {
      v.kind = JVal::Bool;
      i += 5;
      return true;
    }
    if (!s.compare(i, 4, "null")) {
      v.kind = JVal::Null;
      i += 4;
      return true;
    }
    char* end = nullptr;
    v.num = strtod(s.c_str() + i, &end);
    if (end == s.c_str() + i) return fail("unexpected character");
    v.kind = JVal::Num;
    i = end - s.c_str();
    return true;
  }
  bool string(std::string& out) {
    ++i;
    while (i < s.size() && s[i] != '"') {
      if (s[i] == '\\' && i + 1 < s.size()) {
        const char e = s[i + 1];
        out += e == 'n' ? '\n' : e == 't' ? '\t' : e;
        i += 2;
      } else {
        out += s[i++];
      }
    }
    if (i >= s.size()) return fail("unterminated string");
    ++i;
    return true;
  }
  bool array(JVal& v) {
    v.kind = JVal::Arr;
    ++i;
    ws();
    if (i < s.size() && s[i] == ']') {
      ++i;
      return true;
    }
    for (;;) {
      JVal e;
      if (!value(e)) return false;
      v.arr.push_back(std::move(e));
      ws();
      if (i < s.size() && s[i] == ',') {
        ++i;
        continue;
      }
      if (i < s.size() && s[i] == ']') {
        ++i;
        return true;
      }
      return fail("expected , or ]");
    }
  }
  bool object(JVal& v) {
    v.kind = JVal::Obj;
    ++i;
    ws();
    if (i < s.size() && s[i] == '}') {
      ++i;
      return true;
    }
    for (;;) {
      ws();
      if (i >= s.size() || s[i] != '"') return fail("expected a key");
      std::string k;
      if (!string(k)) return false;
      ws();
      if (i >= s.size() || s[i] != ':') return fail("expected :");
      ++i;
      JVal e;
      if (!value(e)) return false;
      v.obj[k] = std::move(e);
      ws();
      if (i < s.size() && s[i] == ',') {
        ++i;
        continue;
      }
      if (i < s.size() && s[i] == '}') {
        ++i;
        return true;
      }
      return fail("expected , or }");
    }
  }
};

double num_or(const JVal& root, const char* k, double def) {
  const JVal* v = root.get(k);
  return v && v->kind == JVal::Num ? v->num : def;
}
std::string str_or(const JVal& root, const char* k, const std::string& def) {
  const JVal* v = root.get(k);
  return v && v->kind == JVal::Str ? v->str : def;
}

int die(const std::string& m) {
  fprintf(stderr, "lightdock_b200: %s\n", m.c_str());
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  std::string file;
  int steps = 100;  // the reference's STEPS on its GPU path
  std::string outdir = ".", resume;
  int device = 0, stop_at = -1;
  int ch;
  const char* usage =
      "usage: lightdock_b200 -f setup.json [-s STEPS] [-o DIR] [-d DEVICE] [-t STOP] [-r CHECKPOINT]";
  while ((ch = getopt(argc, argv, "f:s:l:o:d:r:t:")) != -1) {
    if (ch == 'f') file = optarg;
    else if (ch == 's') steps = atoi(optarg);
    else if (ch == 'l') (void)atoi(optarg);  // parsed and unused, as in the reference
    else if (ch == 'o') outdir = optarg;
    else if (ch == 'd') device = atoi(optarg);
    else if (ch == 'r') resume = optarg;
    else if (ch == 't') stop_at = atoi(optarg);
    else return die(usage);
  }
  if (file.empty()) return die(usage);
  if (steps <= 0) return die("-s STEPS must be positive");
  std::ifstream in(file);
  if (!in) return die("cannot open " + file);
  std::stringstream ss;
  ss << in.rdbuf();
  const std::string text = ss.str();
  JVal root;
  JParser jp(text);
  if (!jp.value(root) || root.kind != JVal::Obj) return die("setup.json: " + (jp.err.empty() ? "not an object" : jp.err));

  const int swarms = (int)num_or(root, "swarms", 0), G = (int)num_or(root, "glowworms", 200);
  const JVal* ua = root.get("use_anm");
  const bool use_anm = !ua || ua->kind != JVal::Bool || ua->b;
  const int anm_rec = use_anm ? (int)num_or(root, "anm_rec", 10) : 0;
  const int anm_lig = use_anm ? (int)num_or(root, "anm_lig", 10) : 0;
  if (swarms <= 0) return die("setup.json: \"swarms\" must be a positive number");
  // the reference CPU path's serial mt19937(0) draws [S][steps][G], made on a host thread while
  // the setup below runs (joined before the first step, or on any early return)
  std::vector<double> u(G > 0 ? (size_t)swarms * steps * G : 0);
  std::thread draws_thread;
  if (G > 0) draws_thread = std::thread([&u, swarms, steps, G]() { sd_gso_draws(0, swarms, steps, G, u.data()); });
  struct Joiner {
    std::thread& t;
    ~Joiner() {
      if (t.joinable()) t.join();
    }
  } draws_joiner{draws_thread};
  const std::string scoring_s = str_or(root, "scoring", "dfire"), prec_s = str_or(root, "precision", "mixed");
  int scoring = scoring_s == "dfire" ? SD_SCORING_DFIRE : scoring_s == "pydock" ? SD_SCORING_PYDOCK : -1;
  if (scoring < 0) return die("setup.json: \"scoring\" must be \"dfire\" or \"pydock\"");
  int precision = prec_s == "mixed" ? SD_PREC_MIXED : prec_s == "fp64" ? SD_PREC_FP64 : prec_s == "fp64_ref" ? SD_PREC_FP64_REF : -1;
  if (precision < 0) return die("setup.json: \"precision\" must be \"mixed\", \"fp64\" or \"fp64_ref\"");
  std::string write_poses = "none";
  double place_secs = 0, anm_secs = 0;
  const int checkpoint_every = (int)num_or(root, "checkpoint_every", 0);
  const JVal* syn = root.get("synthetic");
  const bool pdb_input = !syn || syn->kind != JVal::Obj;
  // PDB inputs: structures read as the reference's setup reads them (flags noxt / noh / now)
  std::unique_ptr<sd_structure, int (*)(sd_structure*)> rec_s(nullptr, sd_structure_free),
      lig_s(nullptr, sd_structure_free);
  if (pdb_input) {
    const std::string rp = str_or(root, "receptor_pdb", ""), lp = str_or(root, "ligand_pdb", "");
    if (rp.empty() || lp.empty())
      return die("setup.json: give receptor_pdb and ligand_pdb, or a \"synthetic\" block");
    auto flag = [&](const char* k) {
      const JVal* v = root.get(k);
      return v && v->kind == JVal::Bool && v->b;
    };
    const int fl = (flag("noxt") ? SD_PDB_NOXT : 0) | (flag("noh") ? SD_PDB_NOH : 0) | (flag("now") ? SD_PDB_NOW : 0);
    auto resolve = [&](const std::string& f) {  // as given, else next to setup.json
      if (std::ifstream(f).good() || f.empty() || f[0] == '/') return f;
      const size_t sl = file.rfind('/');
      return sl == std::string::npos ? f : file.substr(0, sl + 1) + f;
    };
    sd_structure* a = nullptr;
    sd_structure* b = nullptr;
    if (sd_structure_load(resolve(rp).c_str(), fl, &a) != SD_OK) return die(sd_last_error());
    rec_s.reset(a);
    if (sd_structure_load(resolve(lp).c_str(), fl, &b) != SD_OK) return die(sd_last_error());
    lig_s.reset(b);
  }

  sd_synth_spec spec;
  spec.n_swarms = swarms;
  spec.n_glowworms = G;
  spec.n_modes_rec = anm_rec;
  spec.n_modes_lig = anm_lig;
  spec.seed = (unsigned long long)num_or(pdb_input ? root : *syn, "seed", num_or(root, "starting_points_seed", 1));
  if (pdb_input) {
    sd_structure_info(rec_s.get(), &spec.n_rec, nullptr);
    sd_structure_info(lig_s.get(), &spec.n_lig, nullptr);
  } else {
    spec.n_rec = (int)num_or(*syn, "receptor_atoms", 0);
    spec.n_lig = (int)num_or(*syn, "ligand_atoms", 0);
  }
  long long bytes = 0;
  if (sd_synth_buffer_size(&spec, &bytes) != SD_OK) return die(sd_last_error());
  std::unique_ptr<char[]> buf(new char[(size_t)bytes]);
  sd_complex_desc desc;
  double* pos0 = nullptr;
  if (sd_synth_generate(&spec, buf.get(), &desc, &pos0) != SD_OK) return die(sd_last_error());
  if (pdb_input) {
    // real coordinates, masks and DFIRE types; pyDock charges / LJ types stay the seeded
    // stand-ins (charge assignment is a setup stage not built here); swarm placement and
    // starting poses as run_simulation.cc:66-74 places them (before the ANM stage, on the
    // structures as read); ANM modes, which re-centre the structure as cal_anm does; the ligand
    // reference point last, on the final coordinates (prepare_gso_tasks.cc:1201-1202)
    sd_structure_arrays(rec_s.get(), const_cast<double*>(desc.rec_xyz), const_cast<int*>(desc.rec_mask),
                        const_cast<int*>(desc.rec_dfire_type), nullptr, nullptr);
    sd_structure_arrays(lig_s.get(), const_cast<double*>(desc.lig_xyz), const_cast<int*>(desc.lig_mask),
                        const_cast<int*>(desc.lig_dfire_type), nullptr, nullptr);
    write_poses = str_or(root, "write_poses", "representatives");
    if (write_poses != "representatives" && write_poses != "all" && write_poses != "none")
      return die("setup.json: \"write_poses\" must be \"representatives\", \"all\" or \"none\"");
    for (const char* k : {"membrane", "transmembrane", "dense_sampling"}) {
      const JVal* v = root.get(k);
      if (v && v->kind == JVal::Bool && v->b) return die(std::string("setup.json: \"") + k + "\" is not supported");
    }
    const auto p0 = std::chrono::steady_clock::now();
    if (sd_place_swarms(rec_s.get(), lig_s.get(), swarms, G, anm_rec, anm_lig, use_anm ? 1 : 0,
                        (int)num_or(root, "starting_points_seed", 324324), (int)num_or(root, "anm_seed", 324324),
                        num_or(root, "swarm_radius", 10.0), 0, device, nullptr, pos0) != SD_OK)
      return die(sd_last_error());
    const auto p1 = std::chrono::steady_clock::now();
    if (anm_rec > 0 && sd_anm(rec_s.get(), anm_rec, num_or(root, "anm_rec_rmsd", 0.5), swarms, G, device,
                              const_cast<double*>(desc.rec_modes), const_cast<double*>(desc.rec_xyz), nullptr) != SD_OK)
      return die(sd_last_error());
    if (anm_lig > 0 && sd_anm(lig_s.get(), anm_lig, num_or(root, "anm_lig_rmsd", 0.5), swarms, G, device,
                              const_cast<double*>(desc.lig_modes), const_cast<double*>(desc.lig_xyz), nullptr) != SD_OK)
      return die(sd_last_error());
    if (sd_reference_point(desc.lig_xyz, desc.n_lig, desc.lig_ref_point) != SD_OK) return die(sd_last_error());
    const auto p2 = std::chrono::steady_clock::now();
    place_secs = std::chrono::duration<double>(p1 - p0).count();
    anm_secs = std::chrono::duration<double>(p2 - p1).count();
    printf("setup: swarm placement %f s, ANM %f s\n", place_secs, anm_secs);
  }

  const size_t tsz = (size_t)SD_DFIRE_TYPES * SD_DFIRE_TYPES * SD_DFIRE_BINS;
  std::vector<double> table(tsz), eps(SD_LJ_TYPES), sig(SD_LJ_TYPES);
  sd_synth_tables((unsigned long long)num_or(root, "table_seed", 3), table.data(), eps.data(), sig.data());
  const std::string tpath = str_or(root, "dfire_table", "");
  if (!tpath.empty()) {  // DCparams format (prepare_gso_tasks.cc:1175-1189): one value per line
    std::ifstream tf(tpath);
    if (!tf) return die("cannot open dfire_table " + tpath);
    std::string line;
    size_t k = 0;
    while (std::getline(tf, line) && k < tsz) table[k++] = strtod(line.c_str(), nullptr);
    if (k != tsz) return die("dfire_table " + tpath + ": expected 564480 values");
  }
  sd_tables tables = {table.data(), eps.data(), sig.data()};
  sd_gso_params p;
  sd_gso_params_default(&p);
  p.rho = num_or(root, "rho", p.rho);
  p.gamma = num_or(root, "gamma", p.gamma);
  p.beta = num_or(root, "beta", p.beta);
  p.initial_luciferin = num_or(root, "initialLuciferin", p.initial_luciferin);
  p.initial_vision_range = num_or(root, "initialVisionRange", p.initial_vision_range);
  p.max_vision_range = num_or(root, "maximumVisionRange", p.max_vision_range);
  p.max_neighbors = (int)num_or(root, "maximumNeighbors", p.max_neighbors);
  p.translation_step = num_or(root, "translation_step", p.translation_step);
  p.rotation_step = num_or(root, "rotation_step", p.rotation_step);
  p.nmodes_step = num_or(root, "nmodes_step", p.nmodes_step);

  sd_ctx* ctx = nullptr;
  if (sd_ctx_create(&desc, 1, &tables, &p, scoring, precision, device, &ctx) != SD_OK) return die(sd_last_error());
  const auto t0 = std::chrono::steady_clock::now();
  if (draws_thread.joinable()) draws_thread.join();
  const int pl = SD_POSE_LEN(anm_rec, anm_lig);
  const size_t n = (size_t)swarms * G;
  // the whole state, for checkpoints: written to <dir>/checkpoint.ckpt every checkpoint_every steps
  // and at the end; -r resumes from one (same setup), running the remaining steps with their draws
  std::vector<double> kpos(n * pl), ksc(n), kluc(n), kvis(n), kref(n * 3);
  std::vector<int> kstep(n), kmoved(n), knnei(n), ksel(n);
  sd_swarm_state ks = {kpos.data(), ksc.data(), kluc.data(), kvis.data(), kstep.data(),
                       kmoved.data(), knnei.data(), ksel.data(), kref.data()};
  const std::string ckpt_path = (outdir.empty() ? std::string(".") : outdir) + "/checkpoint.ckpt";
  const long long stop = stop_at >= 0 ? std::min(stop_at, steps) : steps;
  if ((checkpoint_every > 0 || !resume.empty() || stop < steps) && !outdir.empty() && outdir != "." &&
      mkdir(outdir.c_str(), 0755) != 0 && errno != EEXIST) {
    sd_ctx_destroy(ctx);
    return die("cannot create output directory " + outdir);
  }
  long long done = 0, resumed_from = 0;
  int rc = SD_OK;
  std::string cli_err;
  if (!resume.empty()) {
    long long planned = 0;
    rc = sd_read_checkpoint(resume.c_str(), swarms, G, pl, &done, &planned, &ks);
    if (!rc && planned != 0 && planned != steps) {
      // the reference's draws [S][STEPS][G] differ with STEPS: only the same run continues
      cli_err = "checkpoint " + resume + " is of a " + std::to_string(planned) + "-step run; give -s " +
                std::to_string(planned);
      rc = SD_ERR_ARG;
    } else if (!rc && done > stop) {
      cli_err = "checkpoint " + resume + " is past step " + std::to_string(stop);
      rc = SD_ERR_ARG;
    }
    if (!rc) rc = sd_set_state(ctx, 0, &ks);
    resumed_from = done;
  } else {
    rc = sd_init_state(ctx, 0, pos0);
  }
  while (!rc && done < stop) {
    const int chunk = (int)std::min<long long>(checkpoint_every > 0 ? checkpoint_every : stop, stop - done);
    std::vector<double> uc((size_t)swarms * chunk * G);  // draws of steps [done, done + chunk)
    for (int sw = 0; sw < swarms; ++sw)
      std::copy(u.begin() + ((size_t)sw * steps + done) * G, u.begin() + ((size_t)sw * steps + done + chunk) * G,
                uc.begin() + (size_t)sw * chunk * G);
    rc = sd_set_draws(ctx, 0, uc.data(), chunk);
    if (!rc) rc = sd_step(ctx, chunk, 1);
    done += chunk;
    if (!rc && (checkpoint_every > 0 || (done == stop && stop < steps))) {
      rc = sd_get_state(ctx, 0, &ks);
      if (!rc) rc = sd_write_checkpoint(ckpt_path.c_str(), swarms, G, pl, done, steps, &ks);
    }
  }
  if (!rc && stop < steps) {  // -t: a segment of the run; the results come with its last segment
    sd_ctx_destroy(ctx);
    printf("stopped after step %lld of %d; resume with -r %s\n", done, steps, ckpt_path.c_str());
    return 0;
  }
  if (rc && !cli_err.empty()) {
    sd_ctx_destroy(ctx);
    return die(cli_err);
  }
  std::vector<double> pos(n * pl), luc(n), vis(n), sc(n);
  std::vector<int> nnei(n);
  sd_swarm_state st = {pos.data(), sc.data(), luc.data(), vis.data(), nullptr, nullptr, nnei.data(), nullptr, nullptr};
  if (!rc) rc = sd_get_state(ctx, 0, &st);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  sd_stats stats = {};
  if (!rc) rc = sd_get_stats(ctx, &stats);
  // PDB inputs: cluster the final poses on their CA / P atoms (cluster.repr per swarm)
  std::vector<int> ncl, crep, clen, cmem;
  double cluster_secs = 0;
  if (!rc && pdb_input) {
    std::vector<int> rbb(desc.n_rec), lbb(desc.n_lig);
    sd_structure_arrays(rec_s.get(), nullptr, nullptr, nullptr, rbb.data(), nullptr);
    sd_structure_arrays(lig_s.get(), nullptr, nullptr, nullptr, lbb.data(), nullptr);
    ncl.resize(swarms);
    crep.resize(n);
    clen.resize(n);
    cmem.resize(n);
    const auto c0 = std::chrono::steady_clock::now();
    rc = sd_cluster(ctx, 0, rbb.data(), lbb.data(), ncl.data(), crep.data(), clen.data(), cmem.data());
    cluster_secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
  }
  auto fail_ctx = [&](const std::string& m) {
    sd_ctx_destroy(ctx);
    return die(m);
  };
  if (rc) return fail_ctx(sd_last_error());
  if (!outdir.empty() && outdir != "." && mkdir(outdir.c_str(), 0755) != 0 && errno != EEXIST)
    return fail_ctx("cannot create output directory " + outdir);
  if (sd_write_gso_output(outdir.c_str(), 0, swarms, G, pl, steps, pos.data(), luc.data(), nnei.data(), vis.data(),
                          sc.data()) != SD_OK)
    return fail_ctx(sd_last_error());
  if (pdb_input && sd_write_cluster_repr(outdir.c_str(), 0, swarms, G, ncl.data(), crep.data(), clen.data(),
                                          sc.data()) != SD_OK)
    return fail_ctx(sd_last_error());
  // PDB inputs: final poses as swarm_<s>/lightdock_<g>.pdb, for the cluster representatives (the
  // files cluster.repr names), every glowworm (as the reference's pipeline writes them), or none
  double pose_secs = 0;
  long long pose_files = 0;
  if (pdb_input && write_poses != "none") {
    const auto w0 = std::chrono::steady_clock::now();
    std::vector<int> which;
    for (int sw = 0; sw < swarms; ++sw) {
      if (write_poses == "all") {
        for (int g = 0; g < G; ++g) which.push_back(sw * G + g);
      } else {
        for (int c = 0; c < ncl[sw]; ++c) which.push_back(sw * G + crep[(size_t)sw * G + c]);
      }
    }
    const size_t per_pose = (size_t)(desc.n_rec + desc.n_lig) * 3;
    const int batch = (int)std::max<size_t>(1, std::min<size_t>(which.size(), ((size_t)256 << 20) / (per_pose * 8)));
    std::vector<double> rx((size_t)batch * desc.n_rec * 3), lx((size_t)batch * desc.n_lig * 3);
    const std::string base = outdir.empty() ? "." : outdir;
    for (size_t k0 = 0; k0 < which.size(); k0 += batch) {
      const int m = (int)std::min<size_t>(batch, which.size() - k0);
      if (sd_materialise_poses(ctx, 0, which.data() + k0, m, rx.data(), lx.data()) != SD_OK)
        return fail_ctx(sd_last_error());
      // the files are independent: format and write them on every host core
      std::atomic<int> next{0}, failed{0};
      std::string first_error;
      std::mutex err_mu;
      auto worker = [&]() {
        for (int k = next++; k < m && !failed; k = next++) {
          const int sw = which[k0 + k] / G, g = which[k0 + k] % G;
          const std::string path =
              base + "/swarm_" + std::to_string(sw) + "/lightdock_" + std::to_string(g) + ".pdb";
          if (sd_write_pose_pdb(path.c_str(), rec_s.get(), rx.data() + (size_t)k * desc.n_rec * 3, lig_s.get(),
                                lx.data() + (size_t)k * desc.n_lig * 3) != SD_OK) {
            std::lock_guard<std::mutex> lk(err_mu);
            if (!failed++) first_error = sd_last_error();
          }
        }
      };
      const int nthreads = (int)std::max(1u, std::min(std::thread::hardware_concurrency(), 64u));
      std::vector<std::thread> pool;
      for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker);
      worker();
      for (auto& th : pool) th.join();
      if (failed) return fail_ctx(first_error);
      pose_files += m;
    }
    pose_secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
  }
  int tv = -1, tw = 0, tb = 0;
  sd_get_tuning(ctx, &tv, &tw, &tb, nullptr, 0);
  sd_ctx_destroy(ctx);
  // the run's figures as one JSON object, <dir>/run.json
  {
    const std::string path = (outdir.empty() ? std::string(".") : outdir) + "/run.json";
    FILE* jf = std::fopen(path.c_str(), "w");
    if (!jf) return die("cannot write " + path);
    std::fprintf(jf,
                 "{\"steps\": %d, \"resumed_from_step\": %lld, \"swarms\": %d, \"glowworms\": %d, "
                 "\"receptor_atoms\": %d, \"ligand_atoms\": %d, \"modes\": [%d, %d], \"scoring\": \"%s\", "
                 "\"precision\": \"%s\", \"seconds\": {\"placement\": %.6f, \"anm\": %.6f, \"gso\": %.6f, "
                 "\"clustering\": %.6f, \"pose_files\": %.6f}, \"scored_poses\": %lld, "
                 "\"scored_poses_per_s\": %.1f, \"pose_files\": %lld, \"mixed_variant\": %d, "
                 "\"counters\": {\"pairs_in_cutoff\": %lld, \"pairs_fallback\": %lld, \"edge_d2_zero\": %lld, "
                 "\"edge_d2_cutoff\": %lld, \"edge_u_zero\": %lld, \"edge_shortfall\": %lld}}\n",
                 steps, resume.empty() ? 0LL : resumed_from, swarms, G, desc.n_rec, desc.n_lig, anm_rec, anm_lig,
                 scoring_s.c_str(), prec_s.c_str(), place_secs, anm_secs, secs, cluster_secs, pose_secs,
                 stats.scored_poses, stats.scored_poses / secs, pose_files, precision == SD_PREC_MIXED ? tv : -1,
                 stats.pairs_in_cutoff, stats.pairs_fallback, stats.edge_d2_zero, stats.edge_d2_cutoff,
                 stats.edge_u_zero, stats.edge_shortfall);
    std::fclose(jf);
  }
  printf("simulation execution:%f\n", secs);
  if (pdb_input) printf("clustering: %f s (cluster.repr per swarm)\n", cluster_secs);
  if (pose_files) printf("pose files: %lld lightdock_<g>.pdb in %f s\n", pose_files, pose_secs);
  printf("scored poses: %lld (%.0f per second, wall clock including setup and state transfers)\n",
         stats.scored_poses, stats.scored_poses / secs);
  return 0;
}
