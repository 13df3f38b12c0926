// Structures from PDB files, as the reference's setup prepares them for the GSO path:
//   read_input_structure / parse_complex_from_file / read_atom_line
//                                  (source/prep/src/read_input_structure.cc:60-307)
//   generate_complex               (source/prep/src/complex.cc:5-123)
//   init_center_translate          (source/prep/src/initialization.cc:3-29)
//   translate                      (source/prep/src/translate.cc)
//   get_nm_mask                    (source/prep/src/complex.cc:143-209)
//   get_docking_model (DFIRE atom types, source/dock/src/prepare_gso_tasks.cc:31-69, tables of
//                      source/dock/include/fastdfire.h)
// Behaviour kept on purpose: coordinates go through float (the reference's Atom stores x, y, z
// as float); the first MODEL only; residues split on (name, number, insertion code); the centre
// is the mean of the non-hydrogen atoms summed in file order (the reference's OpenMP loop has no
// reduction clause, so this is its single-thread result).  Defined here where the reference is
// undefined: an atom without a DFIRE type is an error (the reference indexes its table with an
// uninitialised value); an element it does not recognise is an error (the reference exits); a
// membrane bead (MMB BJ) is an error (the reference's typing skips it without advancing, which
// shifts every later atom's type).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "sd_internal.h"

struct sd_structure {
  std::vector<double> xyz;          // translated (centred) coordinates [n][3]
  std::vector<double> raw_xyz;      // coordinates as read (through float), before centring
  std::vector<int> mask, dfire, backbone;
  std::vector<std::string> atom_name, residue_name, element;
  std::vector<int> residue_first;   // [n_res + 1] first atom of each residue
  // the remaining fields of each atom's record, as read_atom_line keeps them for write_pdb
  std::vector<std::string> record, alt, resname, chain, icode;  // columns 1-6 (untrimmed), 17, 18-21, 22, 27
  std::vector<int> resnum;                             // columns 23-26
  std::vector<float> occupancy, bfactor;               // columns 55-60, 61-66
  double translation[3] = {0, 0, 0};
};

namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r' || s[a] == '\n')) ++a;
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r' || s[b - 1] == '\n')) --b;
  return s.substr(a, b - a);
}

std::string field(const std::string& line, size_t pos, size_t len) {
  if (pos >= line.size()) return std::string();
  return line.substr(pos, len);
}

// occupancy / B-factor as read_atom_line reads them: std::stof of the 6-character field, the
// default when the field is absent, unparsable or not consumed to its end
float numeric_field(const std::string& line, size_t pos, float dflt) {
  try {
    const std::string f = line.substr(pos, 6);
    size_t used = 0;
    const float v = std::stof(f, &used);
    return used < f.size() ? dflt : v;
  } catch (...) {
    return dflt;
  }
}

const char* const kElements[12] = {"C", "N", "O", "H", "S", "P", "CL", "MG", "FE", "PB", "SE", "F"};
bool known_element(const std::string& e) {
  for (const char* k : kElements)
    if (e == k) return true;
  return false;
}

// residues that take part in the normal-mode mask (complex.h STANDARD_TYPES, MODIFIED_TYPES and
// the DNA / RNA standard names)
bool nm_residue(const std::string& r) {
  static const char* const kNames[] = {"ALA", "ARG", "ASN", "ASP", "CYS", "GLU", "GLN", "GLY", "HIS", "ILE",
                                       "LEU", "LYS", "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL",
                                       "CYX", "HIP", "HID", "HIE", "DA",  "DC",  "DI",  "DG",  "DT",  "A",
                                       "C",   "G",   "U",   "I"};
  for (const char* k : kNames)
    if (r == k) return true;
  return false;
}

// DFIRE atom typing: residue index, atom index within the residue, and the 21 x 14 table of
// type numbers (fastdfire.h); the 168 types index the [168][168][20] energy table
int dfire_residue(const std::string& r) {
  static const char* const kRes[21] = {"ALA", "CYS", "ASP", "GLU", "PHE", "GLY", "HIS", "ILE", "LYS", "LEU", "MET",
                                       "ASN", "PRO", "GLN", "ARG", "SER", "THR", "VAL", "TRP", "TYR", "MMB"};
  for (int i = 0; i < 21; ++i)
    if (r == kRes[i]) return i;
  return -1;
}

int dfire_atom(int res, const std::string& a) {
  // atom names of each residue in DFIRE order (backbone N, CA, C, O first)
  static const char* const kAtoms[21][14] = {
      {"N", "CA", "C", "O", "CB"},
      {"N", "CA", "C", "O", "CB", "SG"},
      {"N", "CA", "C", "O", "CB", "CG", "OD1", "OD2"},
      {"N", "CA", "C", "O", "CB", "CG", "CD", "OE1", "OE2"},
      {"N", "CA", "C", "O", "CB", "CG", "CD1", "CD2", "CE1", "CE2", "CZ"},
      {"N", "CA", "C", "O"},
      {"N", "CA", "C", "O", "CB", "CG", "ND1", "CD2", "CE1", "NE2"},
      {"N", "CA", "C", "O", "CB", "CG1", "CG2", "CD1"},
      {"N", "CA", "C", "O", "CB", "CG", "CD", "CE", "NZ"},
      {"N", "CA", "C", "O", "CB", "CG", "CD1", "CD2"},
      {"N", "CA", "C", "O", "CB", "CG", "SD", "CE"},
      {"N", "CA", "C", "O", "CB", "CG", "OD1", "ND2"},
      {"N", "CA", "C", "O", "CB", "CG", "CD"},
      {"N", "CA", "C", "O", "CB", "CG", "CD", "OE1", "NE2"},
      {"N", "CA", "C", "O", "CB", "CG", "CD", "NE", "CZ", "NH1", "NH2"},
      {"N", "CA", "C", "O", "CB", "OG"},
      {"N", "CA", "C", "O", "CB", "OG1", "CG2"},
      {"N", "CA", "C", "O", "CB", "CG1", "CG2"},
      {"N", "CA", "C", "O", "CB", "CG", "CD1", "CD2", "CE2", "NE1", "CE3", "CZ3", "CH2", "CZ2"},
      {"N", "CA", "C", "O", "CB", "CG", "CD1", "CD2", "CE1", "CE2", "CZ", "OH"},
      {"BJ"}};
  if (res < 0 || res >= 21) return -1;
  for (int i = 0; i < 14; ++i)
    if (kAtoms[res][i] && a == kAtoms[res][i]) return i;
  return -1;
}

int dfire_type_of(int res, int atom) {
  static const int kTrans[21][14] = {
      {74, 75, 76, 77, 78},
      {0, 1, 2, 3, 4, 5},
      {122, 123, 124, 125, 126, 127, 128, 129},
      {113, 114, 115, 116, 117, 118, 119, 120, 121},
      {14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24},
      {79, 80, 81, 82},
      {130, 131, 132, 133, 134, 135, 136, 137, 138, 139},
      {25, 26, 27, 28, 29, 30, 31, 32},
      {151, 152, 153, 154, 155, 156, 157, 158, 159},
      {33, 34, 35, 36, 37, 38, 39, 40},
      {6, 7, 8, 9, 10, 11, 12, 13},
      {105, 106, 107, 108, 109, 110, 111, 112},
      {160, 161, 162, 163, 164, 165, 166},
      {96, 97, 98, 99, 100, 101, 102, 103, 104},
      {140, 141, 142, 143, 144, 145, 146, 147, 148, 149, 150},
      {90, 91, 92, 93, 94, 95},
      {83, 84, 85, 86, 87, 88, 89},
      {41, 42, 43, 44, 45, 46, 47},
      {48, 49, 50, 51, 52, 53, 54, 55, 56, 57, 58, 59, 60, 61},
      {62, 63, 64, 65, 66, 67, 68, 69, 70, 71, 72, 73},
      {167}};
  return kTrans[res][atom];
}

}  // namespace

namespace sd {
// atoms of a loaded structure for the setup stages built on it (ANM)
int structure_atoms(const sd_structure* s, std::vector<double>& xyz, std::vector<std::string>& names,
                    std::vector<int>& residue_first) {
  xyz = s->xyz;
  names = s->atom_name;
  residue_first = s->residue_first;
  return SD_OK;
}

const std::vector<double>& structure_raw_xyz(const sd_structure* s) { return s->raw_xyz; }
const std::vector<std::string>& structure_residue_names(const sd_structure* s) { return s->residue_name; }
const std::vector<int>& structure_residue_first(const sd_structure* s) { return s->residue_first; }
const double* structure_translation(const sd_structure* s) { return s->translation; }
}  // namespace sd

extern "C" {

int sd_structure_load(const char* pdb_path, int flags, sd_structure** out) {
  if (!pdb_path || !out) return sd::fail(SD_ERR_ARG, "sd_structure_load: NULL argument");
  *out = nullptr;
  // the reference splits the argument on spaces and uses the first structure's atoms
  std::string path = pdb_path;
  const size_t sp = path.find(' ');
  if (sp != std::string::npos) path = path.substr(0, sp);
  std::ifstream in(path);
  if (!in.is_open()) return sd::fail(SD_ERR_ARG, "sd_structure_load: cannot open " + path);
  const bool noxt = flags & SD_PDB_NOXT, noh = flags & SD_PDB_NOH, now = flags & SD_PDB_NOW;
  sd_structure* s = new sd_structure();
  std::string line, last_res_name = "#", last_ins = "#";
  int last_res_num = 0;
  bool first_residue = true;
  int models = 0;
  std::vector<int> res_count;
  while (std::getline(in, line)) {
    if (models > 1) break;
    const std::string type = trim(field(line, 0, 6));
    if (type == "MODEL") {
      ++models;
      continue;
    }
    if (type != "ATOM" && type != "HETATM") continue;
    if (line.size() < 54) {
      delete s;
      return sd::fail(SD_ERR_ARG, "sd_structure_load: short ATOM line in " + path);
    }
    const std::string name = trim(field(line, 12, 4)), res = trim(field(line, 17, 4));
    const std::string ins = field(line, 26, 1);
    const int res_num = std::atoi(field(line, 22, 4).c_str());
    bool valid = !(now && res == "HOH");
    if ((noh && !name.empty() && name[0] == 'H') || (noxt && name == "OXT")) valid = false;
    if (!valid) continue;
    std::string elem = name.substr(0, std::min<size_t>(2, name.size()));
    if (!known_element(elem)) {
      elem = name.substr(0, std::min<size_t>(1, name.size()));
      if (!known_element(elem)) {
        delete s;
        return sd::fail(SD_ERR_ARG, "sd_structure_load: atom " + name + " has no recognised element");
      }
    }
    // coordinates pass through float, as in the reference's Atom
    for (int k = 0; k < 3; ++k)
      s->xyz.push_back((double)(float)std::strtod(field(line, 30 + 8 * k, 8).c_str(), nullptr));
    s->atom_name.push_back(name);
    s->element.push_back(trim(elem));
    s->record.push_back(line.substr(0, 6));
    s->alt.push_back(trim(field(line, 16, 1)));
    s->resname.push_back(res);
    s->chain.push_back(trim(field(line, 21, 1)));
    s->icode.push_back(ins);
    s->resnum.push_back(res_num);
    s->occupancy.push_back(numeric_field(line, 54, 1.0f));
    s->bfactor.push_back(numeric_field(line, 60, 0.0f));
    if (first_residue || res != last_res_name || res_num != last_res_num || ins != last_ins) {
      first_residue = false;
      last_res_name = res;
      last_res_num = res_num;
      last_ins = ins;
      s->residue_name.push_back(res);
      res_count.push_back(0);
    }
    ++res_count.back();
  }
  const int n = (int)s->atom_name.size();
  if (n == 0) {
    delete s;
    return sd::fail(SD_ERR_ARG, "sd_structure_load: no atoms in " + path);
  }
  s->residue_first.assign(res_count.size() + 1, 0);
  for (size_t r = 0; r < res_count.size(); ++r) s->residue_first[r + 1] = s->residue_first[r] + res_count[r];
  // centre: mean of the non-hydrogen atoms, negated; then translate
  double tx = 0, ty = 0, tz = 0;
  int dim = 0;
  for (int i = 0; i < n; ++i)
    if (s->element[i] != "H") {
      tx += s->xyz[i * 3];
      ty += s->xyz[i * 3 + 1];
      tz += s->xyz[i * 3 + 2];
      ++dim;
    }
  s->raw_xyz = s->xyz;
  s->translation[0] = -1 * tx / dim;
  s->translation[1] = -1 * ty / dim;
  s->translation[2] = -1 * tz / dim;
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) s->xyz[i * 3 + k] += s->translation[k];
  // normal-mode mask, DFIRE types, backbone flags (CA or P, the atoms the clustering compares)
  s->mask.assign(n, 0);
  s->dfire.assign(n, 0);
  s->backbone.assign(n, 0);
  for (size_t r = 0; r + 1 < s->residue_first.size(); ++r) {
    const std::string& rn = s->residue_name[r];
    const int nm = nm_residue(rn) ? 1 : 0;
    const int ri = dfire_residue(rn);
    for (int a = s->residue_first[r]; a < s->residue_first[r + 1]; ++a) {
      s->mask[a] = nm;
      s->backbone[a] = (s->atom_name[a] == "CA" || s->atom_name[a] == "P") ? 1 : 0;
      const int ai = dfire_atom(ri, s->atom_name[a]);
      if (ri < 0 || ai < 0 || rn == "MMB") {
        const std::string what = rn + " " + s->atom_name[a];
        delete s;
        return sd::fail(SD_ERR_ARG, "sd_structure_load: no DFIRE atom type for " + what);
      }
      s->dfire[a] = dfire_type_of(ri, ai);
    }
  }
  *out = s;
  return SD_OK;
}

int sd_structure_info(const sd_structure* s, int* n_atoms, int* n_residues) {
  if (!s) return sd::fail(SD_ERR_ARG, "sd_structure_info: NULL structure");
  if (n_atoms) *n_atoms = (int)s->atom_name.size();
  if (n_residues) *n_residues = (int)s->residue_name.size();
  return SD_OK;
}

int sd_structure_arrays(const sd_structure* s, double* xyz, int* nm_mask, int* dfire_type, int* backbone,
                        double* translation) {
  if (!s) return sd::fail(SD_ERR_ARG, "sd_structure_arrays: NULL structure");
  const size_t n = s->atom_name.size();
  if (xyz) std::memcpy(xyz, s->xyz.data(), n * 3 * sizeof(double));
  if (nm_mask) std::memcpy(nm_mask, s->mask.data(), n * sizeof(int));
  if (dfire_type) std::memcpy(dfire_type, s->dfire.data(), n * sizeof(int));
  if (backbone) std::memcpy(backbone, s->backbone.data(), n * sizeof(int));
  if (translation) std::memcpy(translation, s->translation, 3 * sizeof(double));
  return SD_OK;
}

int sd_structure_free(sd_structure* s) {
  delete s;
  return SD_OK;
}

int sd_write_pose_pdb(const char* path, const sd_structure* receptor, const double* rec_xyz,
                      const sd_structure* ligand, const double* lig_xyz) {
  if (!path || !receptor || !rec_xyz || (!ligand) != (!lig_xyz))
    return sd::fail(SD_ERR_ARG, "sd_write_pose_pdb: bad arguments");
  // left-pad (or right-pad) a field to width w; false where the reference's padding would be
  // negative (it throws there)
  auto pad = [](const std::string& v, size_t w, bool left, std::string& out) {
    if (v.size() > w) return false;
    out += left ? std::string(w - v.size(), ' ') + v : v + std::string(w - v.size(), ' ');
    return true;
  };
  auto fixed = [](double v, int prec) {
    char b[64];
    std::snprintf(b, sizeof b, "%.*f", prec, v);
    return std::string(b);
  };
  std::string text;
  for (int part = 0; part < 2; ++part) {
    const sd_structure* st = part == 0 ? receptor : ligand;
    const double* xyz = part == 0 ? rec_xyz : lig_xyz;
    if (!st) continue;
    for (size_t i = 0; i < st->atom_name.size(); ++i) {
      std::string ln = st->record[i];
      std::string name = st->atom_name[i];
      if (name.size() < 4) name = " " + name;
      bool ok = pad(std::to_string(i + 1), 5, true, ln);
      ln += " ";
      ok = ok && pad(name, 4, false, ln) && pad(st->alt[i], 1, false, ln) &&
           pad(st->resname[i], 3, true, ln) && pad(st->chain[i], 2, true, ln) &&
           pad(std::to_string(st->resnum[i]), 4, true, ln) && pad(st->icode[i], 1, true, ln);
      ln += "   ";
      for (int k = 0; k < 3 && ok; ++k) ok = pad(fixed(xyz[i * 3 + k], 3), 8, true, ln);
      ok = ok && pad(fixed(st->occupancy[i], 2), 6, true, ln) && pad(fixed(st->bfactor[i], 2), 6, true, ln) &&
           pad(st->element[i], 12, true, ln);
      if (!ok)
        return sd::fail(SD_ERR_ARG, "sd_write_pose_pdb: atom " + std::to_string(i + 1) +
                                        " does not fit the PDB columns (serial, residue or coordinate too wide)");
      text += ln;
      text += "\n";
    }
  }
  FILE* f = std::fopen(path, "w");
  if (!f) return sd::fail(SD_ERR_ARG, std::string("sd_write_pose_pdb: cannot open ") + path);
  const bool good = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  if (std::fclose(f) != 0 || !good) return sd::fail(SD_ERR_ARG, std::string("sd_write_pose_pdb: cannot write ") + path);
  return SD_OK;
}

}  // extern "C"
