// Host-side input handling for the grid-map engine: AD4 parameter library,
// GPF/PDBQT loader, lookup tables, H-bond bond vectors, and the .map/.fld/.xyz
// writers.  Compiled with -ffp-contract=off so every double expression rounds
// like the reference's x86-64 build (no fused multiply-adds).
#include "ag_host.h"

#include <algorithm>
#include <memory>
#include <atomic>
#include <chrono>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <thread>

namespace ag {

// 332/eps(r) for the Mehler-Solmajer dielectric (autogrid.h:233-239).
double distDepDielInv(double d) {
  double E = exp(-0.3153767175 * d);
  return (332.0 + (332 * 7.7839) * E) / (78.4 + -66.57180475 * E);
}

// ---------------------------------------------------------------------------
// Log
// ---------------------------------------------------------------------------
Log::~Log() {
  if (own_ && f_) fclose(f_);
}

void Log::open(const char* path) {
  if (path && path[0]) {
    f_ = fopen(path, "w");
    if (!f_) throw ExitProgram{-2, std::string("cannot open log file ") + path};
    own_ = true;
  } else {
    f_ = stdout;
  }
}

void Log::print(const char* fmt, ...) {
  if (!f_) return;
  va_list ap;
  va_start(ap, fmt);
  vfprintf(f_, fmt, ap);
  va_end(ap);
}

void Log::warn(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (f_) fprintf(f_, "%s: WARNING:  %s\n", programName.c_str(), buf);
  // Echo the first few to stderr like the reference; synthetic receptors can trigger thousands.
  if (++nWarn_ <= 10) fprintf(stderr, "%s: WARNING:  %s\n", programName.c_str(), buf);
  else if (nWarn_ == 11) fprintf(stderr, "%s: further warnings go to the log only\n", programName.c_str());
}

void Log::fatal(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (f_) fprintf(f_, "%s: ERROR: %s\n", programName.c_str(), buf);
  fprintf(stderr, "%s: ERROR: %s\n", programName.c_str(), buf);
  throw ExitProgram{code, buf};
}

// ---------------------------------------------------------------------------
// Parameter library (ParameterLibrary.cpp:34-234)
// ---------------------------------------------------------------------------
namespace {

// The two built-in AD4 parameter sets, in the AD4 .dat text format.  Only the
// free-energy coefficients differ between them; the atom_par records are the
// same physical constants in both (autodock/default_parameters.h).
const char* const kFE40[] = {"FE_coeff_vdW    0.1560", "FE_coeff_hbond  0.0974",
                             "FE_coeff_estat  0.1465", "FE_coeff_desolv 0.1159",
                             "FE_coeff_tors   0.2744"};
const char* const kFE41[] = {"FE_coeff_vdW    0.1662", "FE_coeff_hbond  0.1209",
                             "FE_coeff_estat  0.1406", "FE_coeff_desolv 0.1322",
                             "FE_coeff_tors   0.2983"};
// type  Rii  epsii  vol  solpar  Rij_hb  epsij_hb  hbond  rec  map  bond
const char* const kAtomPar[] = {
    "atom_par H      2.00  0.020   0.0000   0.00051  0.0  0.0  0  -1  -1  3",
    "atom_par HD     2.00  0.020   0.0000   0.00051  0.0  0.0  2  -1  -1  3",
    "atom_par HS     2.00  0.020   0.0000   0.00051  0.0  0.0  1  -1  -1  3",
    "atom_par C      4.00  0.150  33.5103  -0.00143  0.0  0.0  0  -1  -1  0",
    "atom_par A      4.00  0.150  33.5103  -0.00052  0.0  0.0  0  -1  -1  0",
    "atom_par N      3.50  0.160  22.4493  -0.00162  0.0  0.0  0  -1  -1  1",
    "atom_par NA     3.50  0.160  22.4493  -0.00162  1.9  5.0  4  -1  -1  1",
    "atom_par NS     3.50  0.160  22.4493  -0.00162  1.9  5.0  3  -1  -1  1",
    "atom_par OA     3.20  0.200  17.1573  -0.00251  1.9  5.0  5  -1  -1  2",
    "atom_par OS     3.20  0.200  17.1573  -0.00251  1.9  5.0  3  -1  -1  2",
    "atom_par F      3.09  0.080  15.4480  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Mg     1.30  0.875   1.5600  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par MG     1.30  0.875   1.5600  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par P      4.20  0.200  38.7924  -0.00110  0.0  0.0  0  -1  -1  5",
    "atom_par SA     4.00  0.200  33.5103  -0.00214  2.5  1.0  5  -1  -1  6",
    "atom_par S      4.00  0.200  33.5103  -0.00214  0.0  0.0  0  -1  -1  6",
    "atom_par Cl     4.09  0.276  35.8235  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par CL     4.09  0.276  35.8235  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Ca     1.98  0.550   2.7700  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par CA     1.98  0.550   2.7700  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Mn     1.30  0.875   2.1400  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par MN     1.30  0.875   2.1400  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Fe     1.30  0.010   1.8400  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par FE     1.30  0.010   1.8400  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Zn     1.48  0.550   1.7000  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par ZN     1.48  0.550   1.7000  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Br     4.33  0.389  42.5661  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par BR     4.33  0.389  42.5661  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par I      4.72  0.550  55.0585  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Z      4.00  0.150  33.5103  -0.00143  0.0  0.0  0  -1  -1  0",
    "atom_par G      4.00  0.150  33.5103  -0.00143  0.0  0.0  0  -1  -1  0",
    "atom_par GA     4.00  0.150  33.5103  -0.00052  0.0  0.0  0  -1  -1  0",
    "atom_par J      4.00  0.150  33.5103  -0.00143  0.0  0.0  0  -1  -1  0",
    "atom_par Q      4.00  0.150  33.5103  -0.00143  0.0  0.0  0  -1  -1  0",
};

// Keyword of a parameter-file line: the first token, lowercased, matched as a
// prefix of the known keywords (ParameterLibrary.cpp:241-284).
enum ParTok { PAR_UNKNOWN = -1, PAR_NULL = 0, PAR_VDW, PAR_HBOND, PAR_ESTAT, PAR_DESOLV, PAR_TORS, PAR_ATOM_PAR, PAR_COMMENT };

ParTok parseParamLine(const char* line) {
  char c[512];
  int j = 0;
  for (; line[j] && line[j] != ' ' && line[j] != '\t' && line[j] != '\n' && j < 511; j++)
    c[j] = (char)tolower((unsigned char)line[j]);
  c[j] = 0;
  if (j == 0 && (line[0] == '\n' || line[0] == '\0')) return PAR_NULL;
  if (c[0] == '#') return PAR_COMMENT;
  static const struct { const char* lex; ParTok tok; } table[] = {
      {"FE_coeff_vdW", PAR_VDW},   {"FE_coeff_hbond", PAR_HBOND}, {"FE_coeff_estat", PAR_ESTAT},
      {"FE_coeff_desolv", PAR_DESOLV}, {"FE_coeff_tors", PAR_TORS}, {"atom_par", PAR_ATOM_PAR}};
  if (j == 0) return PAR_NULL;
  ParTok tok = PAR_UNKNOWN;
  for (auto& t : table)
    if (tok == PAR_UNKNOWN && strncasecmp(t.lex, c, j) == 0) tok = t.tok;
  return tok;
}

}  // namespace

ParamLib::ParamLib(bool version4) : slot_(65536, -1) {
  for (const char* l : (version4 ? kFE40 : kFE41)) readLine(l);
  for (const char* l : kAtomPar) readLine(l);
}

unsigned ParamLib::hashKey(const char* key) {
  size_t n = strlen(key);
  if (n == 0) return 0;
  if (n == 1) return (unsigned)(int)key[0] & 0xFFFFu;
  return ((unsigned)(int)key[0] + 256u * (unsigned)(int)key[1]) & 0xFFFFu;
}

AtomParam* ParamLib::find(const char* key) {
  int s = slot_[hashKey(key)];
  return s < 0 ? nullptr : &entries_[s];
}
const AtomParam* ParamLib::find(const char* key) const {
  int s = slot_[hashKey(key)];
  return s < 0 ? nullptr : &entries_[s];
}
int ParamLib::recIndexOf(const char* key) const {
  const AtomParam* a = find(key);
  return a ? a->recIndex : -1;
}

void ParamLib::readLine(const char* line) {
  switch (parseParamLine(line)) {
    case PAR_VDW: sscanf(line, "%*s %lf", &coeff_vdW); break;
    case PAR_HBOND: sscanf(line, "%*s %lf", &coeff_hbond); break;
    case PAR_ESTAT: sscanf(line, "%*s %lf", &coeff_estat); break;
    case PAR_DESOLV: sscanf(line, "%*s %lf", &coeff_desolv); break;
    case PAR_TORS: sscanf(line, "%*s %lf", &coeff_tors); break;
    case PAR_ATOM_PAR: {
      AtomParam a;
      int hb = 0;
      char type[64] = {0};
      int nf = sscanf(line, "%*s %63s %lf %lf %lf %lf %lf %lf %d %d %d %d", type, &a.Rij, &a.epsij, &a.vol,
                      &a.solpar, &a.RijHB, &a.epsijHB, &hb, &a.recIndex, &a.mapIndex, &a.bondIndex);
      if (nf < 2) return;
      strncpy(a.type, type, 7);
      a.hbond = (hb <= A2) ? hb : NON;
      a.epsij *= coeff_vdW;
      a.epsijHB *= coeff_hbond;
      unsigned h = hashKey(a.type);
      if (slot_[h] < 0) {
        slot_[h] = (int)entries_.size();
        entries_.push_back(a);
      } else {
        entries_[slot_[h]] = a;
      }
      break;
    }
    default: break;
  }
}

void ParamLib::loadFile(const char* path) {
  FILE* f = fopen(path, "r");
  if (!f) throw ExitProgram{-1, std::string("Sorry, I can't find or open ") + path};
  char line[256];
  while (fgets(line, sizeof line, f)) readLine(line);
  fclose(f);
}

// ---------------------------------------------------------------------------
// GPF / PDBQT loader (InputDataLoader.cpp:100-797)
// ---------------------------------------------------------------------------
namespace {

enum GpfTok {
  G_UNKNOWN = -1, G_NULL = 0, G_COMMENT, G_RECEPTOR, G_GRIDFLD, G_NPTS, G_SPACING, G_GRIDCENTER,
  G_LIGAND_TYPES, G_MAP, G_NBP_COEFFS, G_NBP_R_EPS, G_ELECMAP, G_DIEL, G_FMAP, G_DISORDER,
  G_SMOOTH, G_SOL_PAR, G_CONSTANT, G_COVALENTMAP, G_RECEPTOR_TYPES, G_PARAM_FILE, G_DSOLVMAP, G_QASP
};

// The keyword is everything up to the first space (or tab), lowercased, and is
// matched by prefix in a fixed order (InputDataLoader.cpp:799-865).
GpfTok parseGpfLine(const char* line) {
  const char* sp = strchr(line, ' ');
  if (!sp) sp = strchr(line, '\t');
  size_t l = sp ? (size_t)(sp - line) : strlen(line);
  char c[512];
  size_t i = 0;
  for (; i < l && i < 511; i++) c[i] = (char)tolower((unsigned char)line[i]);
  c[i] = 0;
  if (c[0] == '\n' || c[0] == '\0' || c[0] == '\r') return G_NULL;
  if (c[0] == '#') return G_COMMENT;
  static const struct { const char* kw; size_t n; GpfTok tok; } kws[] = {
      {"receptor_types", 14, G_RECEPTOR_TYPES}, {"receptor", 8, G_RECEPTOR}, {"gridfld", 7, G_GRIDFLD},
      {"npts", 4, G_NPTS}, {"spacing", 7, G_SPACING}, {"gridcenter", 10, G_GRIDCENTER},
      {"types", 5, G_LIGAND_TYPES}, {"ligand_types", 12, G_LIGAND_TYPES}, {"map", 3, G_MAP},
      {"elecmap", 7, G_ELECMAP}, {"dsolvmap", 8, G_DSOLVMAP}, {"covalentmap", 11, G_COVALENTMAP},
      {"nbp_coeffs", 10, G_NBP_COEFFS}, {"nbp_r_eps", 9, G_NBP_R_EPS}, {"dielectric", 10, G_DIEL},
      {"qasp", 4, G_QASP}, {"fmap", 4, G_FMAP}, {"disorder_h", 10, G_DISORDER}, {"smooth", 6, G_SMOOTH},
      {"sol_par", 7, G_SOL_PAR}, {"constant", 8, G_CONSTANT}, {"parameter_file", 14, G_PARAM_FILE}};
  for (auto& k : kws)
    if (strncmp(c, k.kw, k.n) == 0) return k.tok;
  return G_UNKNOWN;
}

// Whitespace-separated words after the keyword, at most maxwords
// (InputDataLoader.cpp:869-917).
std::vector<std::string> parseTypes(const char* line, int maxwords) {
  std::vector<std::string> out;
  const char* p = line;
  bool keyword = false;
  for (;;) {
    while (*p && isspace((unsigned char)*p)) p++;
    if (!*p) return out;
    const char* s = p;
    while (*p && !isspace((unsigned char)*p)) p++;
    if (!keyword) keyword = true;
    else out.emplace_back(s, p - s);
    if (!*p) return out;
    p++;
    if ((int)out.size() >= maxwords) return out;
  }
}

// npts must be positive, even and at most 1024 (InputDataLoader.cpp:868-887).
int checkSize(int npts, char axis, Log& log) {
  if (npts < 0) log.fatal(-2, "Negative number of %c-grid elements!  Aborting.", axis);
  if (npts == 0) log.warn("0 %c-grid elements!", axis);
  else if (npts > kMaxGridPts) {
    log.warn("Maximum number of %c-grid elements allowed is %d. Using this value.", axis, kMaxGridPts);
    npts = kMaxGridPts;
  } else if (npts % 2 == 1) {
    log.print("Number of grid elements must be even; %c-elements changed to: %d\n", axis, npts);
    npts -= 1;
  }
  return npts;
}


void readReceptor(Problem& p, ParamLib& lib, Log& log, const char* fname, bool hasTypesLine,
                  int typesLineCount, double cmean[3]) {
  FILE* f = fopen(fname, "r");
  if (!f) log.fatal(-2, "can't find or open receptor PDBQT file \"%s\".", fname);
  p.charge.clear(); p.vol.clear(); p.solpar.clear(); p.atomType.clear(); p.hbond.clear(); p.xyzw.clear();
  double csum[3] = {0, 0, 0};
  double qmax = -kBig, qmin = kBig, qtot = 0;
  char line[256];
  int ia = 0;
  while (fgets(line, sizeof line, f)) {
    char record[16] = {0};
    sscanf(line, "%6s", record);
    if (strncmp(record, "ATOM", 4) && strncmp(record, "HETA", 4) && strncmp(record, "CHAR", 4)) continue;
    size_t len = strlen(line);
    double x = 0, y = 0, z = 0, q = 0;
    char type[64] = {0};
    if (len > 30) sscanf(&line[30], "%lf", &x);
    if (len > 38) sscanf(&line[38], "%lf", &y);
    if (len > 46) sscanf(&line[46], "%lf", &z);
    if (len > 70) sscanf(&line[70], "%lf", &q);
    if (len > 77) sscanf(&line[77], "%63s", type);
    AtomParam* a = lib.find(type);
    if (!a) {
      log.print("\n\nreceptor file contains unknown type: '%s'\nadd parameters for it to the parameter library first\n", type);
      fclose(f);
      throw ExitProgram{-1, std::string("receptor file contains unknown type: ") + type};
    }
    if (a->recIndex < 0) {
      strncpy(p.receptorTypes[p.numReceptorTypes], a->type, 2);
      p.receptorTypes[p.numReceptorTypes][2] = 0;
      a->recIndex = p.numReceptorTypes++;
    }
    p.atomType.push_back(a->recIndex);
    p.solpar.push_back(a->solpar);
    p.vol.push_back(a->vol);
    p.hbond.push_back(a->hbond);
    p.charge.push_back(q);
    p.xyzw.insert(p.xyzw.end(), {x, y, z, 0.0});
    qmax = std::max(qmax, q);
    qmin = std::min(qmin, q);
    csum[0] += x; csum[1] += y; csum[2] += z;
    qtot += q;
    ia++;
  }
  fclose(f);
  if (hasTypesLine && p.numReceptorTypes != typesLineCount)
    log.fatal(-2, "The number of atom types found in the receptor PDBQT (%d) does not match the number specified by the \"receptor_types\" command (%d) in the GPF!",
              p.numReceptorTypes, typesLineCount);
  p.numAtoms = ia;
  log.print("\nReceptor Input File :\t%s\n", fname);
  log.print("\nMaximum partial atomic charge found = %+.3lf e\n", qmax);
  log.print("Minimum partial atomic charge found = %+.3lf e\n\n", qmin);
  if (qmax == 0 && qmin == 0)
    log.fatal(-2, "No partial atomic charges were found in the receptor PDBQT file %s!", fname);
  log.print("\nTotal number of atoms :\t\t%d atoms \nTotal charge :\t\t\t%.2lf e\n", ia, qtot);
  for (int k = 0; k < 3; k++) cmean[k] = csum[k] / ia;
}

}  // namespace

void loadGPF(Problem& p, ParamLib& lib, Log& log, const char* gpfPath) {
  FILE* gpf = stdin;
  if (gpfPath && gpfPath[0]) {
    gpf = fopen(gpfPath, "r");
    if (!gpf) {
      fprintf(stderr, "%s: ERROR: Sorry, I can't find or open Grid Parameter File \"%s\"\n", log.programName.c_str(), gpfPath);
      throw ExitProgram{911, std::string("can't find or open Grid Parameter File ") + gpfPath};
    }
  }
  p.gpfName = gpfPath ? gpfPath : "";
  double cmean[3] = {0, 0, 0};
  bool hasTypesLine = false;
  int typesLineCount = 0;
  int mapIndex = -1;
  FILE* xyzf = nullptr;
  double diel = 0;
  char line[256];

  while (fgets(line, sizeof line, gpf)) {
    GpfTok tok = parseGpfLine(line);
    log.print("GPF> %s", line);
    if (tok == G_UNKNOWN) {
      log.warn("Unrecognized keyword in grid parameter file.");
      continue;
    }
    if (tok != G_NULL && tok != G_COMMENT) {
      char* hash = strchr(line, '#');
      if (hash) *hash = 0;
    }
    char tokbuf[256] = {0};
    switch (tok) {
      case G_RECEPTOR:
        sscanf(line, "%*s %255s", tokbuf);
        p.receptorFilename = tokbuf;
        readReceptor(p, lib, log, tokbuf, hasTypesLine, typesLineCount, cmean);
        break;
      case G_GRIDFLD: {
        sscanf(line, "%*s %255s", tokbuf);
        p.fldFilename = tokbuf;
        const char* pos = strstr(tokbuf, ".fld");
        if (!pos) log.fatal(-2, "Grid data file needs the extension \".fld\" for AVS input");
        std::string xyz = tokbuf;
        size_t at = xyz.find("fld");
        xyz.replace(at, 3, "xyz");
        p.xyzFilename = xyz;
        if (xyzf) fclose(xyzf);
        xyzf = fopen(xyz.c_str(), "w");
        if (!xyzf) log.fatal(-2, "can't create grid extrema data file %s", xyz.c_str());
        break;
      }
      case G_NPTS: {
        int m[3] = {0, 0, 0};
        sscanf(line, "%*s %d %d %d", &m[0], &m[1], &m[2]);
        for (int i = 0; i < 3; i++) {
          m[i] = checkSize(m[i], "xyz"[i], log);
          p.n2[i] = m[i] / 2;
          p.n[i] = m[i] + 1;
        }
        p.numPoints = (int64_t)p.n[0] * p.n[1] * p.n[2];
        p.nptsSet = true;
        break;
      }
      case G_SPACING: sscanf(line, "%*s %lf", &p.spacing); break;
      case G_GRIDCENTER: {
        sscanf(line, "%*s %255s", tokbuf);
        if (strncmp(tokbuf, "auto", 4) == 0) {
          for (int k = 0; k < 3; k++) p.center[k] = cmean[k];
        } else {
          sscanf(line, "%*s %lf %lf %lf", &p.center[0], &p.center[1], &p.center[2]);
        }
        for (int ia = 0; ia < p.numAtoms; ia++)
          for (int k = 0; k < 3; k++) p.xyzw[4 * ia + k] -= p.center[k];
        for (int k = 0; k < 3; k++) {
          double ext = p.n2[k] * p.spacing;
          p.cornerMax[k] = p.center[k] + ext;
          p.cornerMin[k] = p.center[k] - ext;
        }
        if (!xyzf) log.fatal(-2, "\"gridfld\" must precede \"gridcenter\" in the GPF");
        for (int k = 0; k < 3; k++) fprintf(xyzf, "%.3lf %.3lf\n", p.cornerMin[k], p.cornerMax[k]);
        fclose(xyzf);
        xyzf = nullptr;
        break;
      }
      case G_LIGAND_TYPES: {
        std::vector<std::string> types = parseTypes(line, kMaxAtomTypes);
        for (size_t i = 0; i < types.size(); i++) {
          AtomParam* a = lib.find(types[i].c_str());
          if (!a) {
            log.print("unknown ligand atom type %s\nadd parameters for it to the parameter library first!\n", types[i].c_str());
            throw ExitProgram{-1, "unknown ligand atom type " + types[i]};
          }
          a->mapIndex = (int)i;
        }
        p.maps.assign(types.size(), MapSpec());
        p.mapsDeclared = true;
        if (!p.nptsSet)
          log.fatal(-2, "You need to set the number of grid points using \"npts\" before setting the ligand atom types, using \"ligand_types\".");
        for (size_t i = 0; i < types.size(); i++) {
          MapSpec& g = p.maps[i];
          strncpy(g.type, types[i].c_str(), 2);
          g.type[2] = 0;
          const AtomParam* a = lib.find(types[i].c_str());
          if (types[i] == "Z") g.isCovalent = true;
          g.solparProbe = a->solpar;
          g.volProbe = a->vol;
          g.Rij = a->Rij;
          g.epsij = a->epsij;
          g.hbond = a->hbond;
          g.RijHB = a->RijHB;
          g.epsijHB = a->epsijHB;
          if (g.hbond > 0) g.isHBonder = true;
          for (int j = 0; j < p.numReceptorTypes; j++) {
            const AtomParam* r = lib.find(p.receptorTypes[j]);
            g.nbpR[j] = (g.Rij + r->Rij) / 2;
            g.nbpEps[j] = sqrt(g.epsij * r->epsij);
            g.xA[j] = 12;
            g.xB[j] = 6;
            g.hbonder[j] = 0;
            if (g.hbond > D1 && (r->hbond == DS || r->hbond == D1)) {
              g.xB[j] = 10; g.hbonder[j] = 1; g.isHBonder = true;
              g.nbpR[j] = g.RijHB; g.nbpEps[j] = g.epsijHB;
            } else if ((g.hbond == DS || g.hbond == D1) && r->hbond > D1) {
              g.xB[j] = 10; g.hbonder[j] = 1; g.isHBonder = true;
              g.nbpR[j] = r->RijHB; g.nbpEps[j] = r->epsijHB;
            }
          }
        }
        break;
      }
      case G_RECEPTOR_TYPES: {
        std::vector<std::string> types = parseTypes(line, kMaxAtomTypes);
        p.numReceptorTypes = (int)types.size();
        typesLineCount = p.numReceptorTypes;
        hasTypesLine = true;
        for (size_t i = 0; i < types.size(); i++) {
          strncpy(p.receptorTypes[i], types[i].c_str(), 2);
          p.receptorTypes[i][2] = 0;
        }
        for (size_t i = 0; i < types.size(); i++) {
          AtomParam* a = lib.find(types[i].c_str());
          if (!a) log.fatal(-2, "Unknown receptor type: \"%s\"", types[i].c_str());
          a->recIndex = (int)i;
        }
        break;
      }
      case G_SOL_PAR: {
        char t[64] = {0};
        double v = 0, s = 0;
        sscanf(line, "%*s %63s %lf %lf", t, &v, &s);
        AtomParam* a = lib.find(t);
        if (a) {
          a->vol = v;
          a->solpar = s;
          if (a->mapIndex >= 0 && a->mapIndex < (int)p.maps.size()) p.maps[a->mapIndex].solparProbe = s;
        }
        break;
      }
      case G_MAP:
        ++mapIndex;
        if (mapIndex >= (int)p.maps.size())
          log.fatal(-2, "Too many \"map\" keywords (%d);  the \"ligand_types\" command declares only %d atom types.",
                    mapIndex + 1, (int)p.maps.size());
        sscanf(line, "%*s %255s", tokbuf);
        p.maps[mapIndex].filename = tokbuf;
        break;
      case G_ELECMAP: sscanf(line, "%*s %255s", tokbuf); p.elecFilename = tokbuf; break;
      case G_DSOLVMAP: sscanf(line, "%*s %255s", tokbuf); p.desolvFilename = tokbuf; break;
      case G_COVALENTMAP: {
        double hw = 1.0;
        sscanf(line, "%*s %lf %lf %lf %lf %lf", &hw, &p.covBarrier, &p.covalentPoint[0], &p.covalentPoint[1], &p.covalentPoint[2]);
        p.covHalfWidthSquaredInv = 1 / (hw * hw);
        for (int k = 0; k < 3; k++) p.covalentPoint[k] -= p.center[k];
        break;
      }
      case G_DISORDER: p.disorderH = true; break;
      case G_SMOOTH: sscanf(line, "%*s %lf", &p.rSmooth); break;
      case G_QASP: sscanf(line, "%*s %lf", &p.solparQ); break;
      case G_DIEL:
        sscanf(line, "%*s %lf", &diel);
        if (diel < 0) {
          p.distDepDiel = true;
          p.epsilon.assign(kMaxDist, 0.0);
          for (int i = 0; i < kMaxDist; i++) p.epsilon[i] = distDepDielInv(double(i) * (1 / 100.0));
        } else {
          p.distDepDiel = false;
          if (diel <= kApproxZero) diel = 40;
          p.invDielCal = 332 / diel;
        }
        break;
      case G_FMAP: sscanf(line, "%*s %255s", tokbuf); p.floatingGridFilename = tokbuf; break;
      case G_PARAM_FILE: sscanf(line, "%*s %255s", tokbuf); p.parameterLibraryFilename = tokbuf; break;
      default: break;
    }
  }
  if (gpf != stdin) fclose(gpf);
  if (xyzf) fclose(xyzf);

  if (!p.mapsDeclared) log.fatal(-2, "No \"ligand_types\" line found in the GPF.");
  if (mapIndex < (int)p.maps.size() - 1) log.fatal(-2, "Not enough map keywords found.");
  if (p.desolvFilename.empty()) log.fatal(-2, "No desolvation map file defined.");
  if (p.elecFilename.empty()) log.fatal(-2, "No electrostatic map file defined.");
  if (p.numAtoms == 0) log.fatal(-2, "No receptor atoms were read.");

  for (int ia = 0; ia < p.numAtoms; ia++)
    p.xyzw[4 * ia + 3] = p.distDepDiel ? p.charge[ia] * lib.coeff_estat
                                       : p.charge[ia] * lib.coeff_estat * p.invDielCal;
}

// ---------------------------------------------------------------------------
// Tables and bond vectors
// ---------------------------------------------------------------------------
namespace {

// 12-6 / 12-10 pair energies in 0.01 A bins with the min-smoothing window
// (PairwiseInteractionEnergies.cpp:36-138).
void energyTables(Problem& p) {
  const int nm = p.numMaps(), nt = p.numReceptorTypes;
  p.energy.assign((size_t)std::max(nt, 1) * kMaxDist * std::max(nm, 1), 0.0);
  auto at = [&](int t, int i, int m) -> double& { return p.energy[((size_t)t * kMaxDist + i) * nm + m]; };
  int iSmooth = int(p.rSmooth * 100 / 2);
  std::vector<double> smooth(kMaxDist);
  for (int m = 0; m < nm; m++) {
    const MapSpec& g = p.maps[m];
    if (g.isCovalent) continue;
    for (int t = 0; t < nt; t++) {
      int xA = g.xA[t], xB = g.xB[t];
      double Rij = g.nbpR[t], epsij = g.nbpEps[t];
      double tmp = epsij / (xA - xB);
      double cA = tmp * pow(Rij, xA) * xB;
      double cB = tmp * pow(Rij, xB) * xA;
      double dxA = xA, dxB = xB;
      for (int i = 1; i < kMaxDist; i++) {
        double r = double(i) * (1 / 100.0);
        double rA = pow(r, dxA), rB = pow(r, dxB);
        double e = cA / rA - cB / rB;
        at(t, i, m) = (kEintClamp < e) ? kEintClamp : e;
      }
      at(t, 0, m) = kEintClamp;
      at(t, kMaxDist - 1, m) = 0;
      if (iSmooth > 0) {
        for (int i = 1; i < kMaxDist; i++) {
          double s = 100000;
          for (int j = std::max(0, i - iSmooth); j < std::min(kMaxDist, i + iSmooth); j++) s = std::min(s, at(t, j, m));
          smooth[i] = s;
        }
        for (int i = 1; i < kMaxDist; i++) at(t, i, m) = smooth[i];
      }
    }
  }
}

// Desolvation Gaussian (DesolvExpFunc.cpp:27-43).  Entry 0 is left at zero, the
// value AutoGrid 4.2.1 has there (its table is a zero-initialised static).
void desolvTable(Problem& p, double coeffDesolv) {
  p.sol.assign(kMaxDist, 0.0);
  double sigma = 3.6;
  double k = -1 / (2 * sigma * sigma);
  for (int i = 1; i < kMaxDist; i++) {
    double r = double(i) * (1 / 100.0);
    p.sol[i] = exp((r * r) * k);
    p.sol[i] *= coeffDesolv;
  }
}

struct V3 { double x, y, z; };
inline V3 pos(const Problem& p, int i) { return {p.xyzw[4 * i], p.xyzw[4 * i + 1], p.xyzw[4 * i + 2]}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 mul(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 divs(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double mag2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double rsqrtd(double a) { return 1 / sqrt(a); }
inline V3 normalized(V3 v) {
  double rd2 = mag2(v);
  if (rd2 < kApproxZero) rd2 = kApproxZero;
  return mul(v, rsqrtd(rd2));
}

// Per-atom geometry of directional H-bonds from covalent partners found among
// the 20 atoms before and after in file order (BondVectors.cpp:45-393).  Atoms
// for which the reference leaves a vector unset get a zero vector here.
void bondVectors(Problem& p, const ParamLib& lib, Log& log) {
  const int N = p.numAtoms;
  p.disorder.assign(N, 0);
  p.rexp.assign(N, 0);
  p.rvector.assign(3 * (size_t)N, 0.0);
  p.rvector2.assign(3 * (size_t)N, 0.0);
  auto setv = [&](std::vector<double>& v, int i, V3 a) { v[3 * i] = a.x; v[3 * i + 1] = a.y; v[3 * i + 2] = a.z; };
  auto getv = [&](const std::vector<double>& v, int i) { return V3{v[3 * i], v[3 * i + 1], v[3 * i + 2]}; };
  const int hydrogen = lib.recIndexOf("HD"), nonHBhydrogen = lib.recIndexOf("H");
  const int carbon = lib.recIndexOf("C"), aromCarbon = lib.recIndexOf("A");
  const int oxygen = lib.recIndexOf("OA"), sulphur = lib.recIndexOf("SA");
  int i1 = 0, i2 = 0, i3 = 0;  // persist across atoms like the reference's locals
  for (int ia = 0; ia < N; ia++) {
    int from = std::max(ia - 20, 0), to = std::min(ia + 20, N - 1);
    const int* T = p.atomType.data();
    if (p.hbond[ia] == D1) {
      for (int ib = from; ib <= to; ib++) {
        if (ib == ia) continue;
        V3 d = sub(pos(p, ia), pos(p, ib));
        double rd2 = mag2(d);
        if (rd2 < 1.90) {
          if (rd2 < kApproxZero) rd2 = kApproxZero;
          double inv = rsqrtd(rd2);
          if (T[ib] != oxygen && T[ib] != sulphur) p.rexp[ia] = 2;
          if (T[ib] == oxygen || T[ib] == sulphur) {
            p.rexp[ia] = 4;
            if (p.disorderH) p.disorder[ia] = 1;
          }
          setv(p.rvector, ia, mul(d, inv));
          break;
        }
      }
    } else if (p.hbond[ia] == A2) {
      int nbond = 0;
      int ib = from;
      for (; ib <= to; ib++) {
        if (ib == ia) continue;
        double rd2 = mag2(sub(pos(p, ia), pos(p, ib)));
        bool isH = T[ib] == hydrogen || T[ib] == nonHBhydrogen;
        if ((rd2 < 3.61 && !isH) || (rd2 < 1.69 && isH)) {
          if (nbond == 2) log.warn("Found an H-bonding atom with three bonded atoms, atom serial number %d", ia + 1);
          if (nbond == 1) { nbond = 2; i2 = ib; }
          if (nbond == 0) { nbond = 1; i1 = ib; }
        }
      }
      if (nbond == 0)
        log.warn("Oxygen atom found with no bonded atoms, atom serial number %d, input->atomType %d", ia + 1, T[ia]);
      if (nbond == 1) {
        setv(p.rvector, ia, normalized(sub(pos(p, ia), pos(p, i1))));
        for (int j2 = from; j2 <= to; j2++) {
          if (j2 == i1 || j2 == ia) continue;
          double rd2 = mag2(sub(pos(p, i1), pos(p, j2)));
          if ((rd2 < 2.89 && T[j2] != hydrogen) || (rd2 < 1.69 && T[j2] == hydrogen)) {
            V3 d = normalized(sub(pos(p, j2), pos(p, i1)));
            setv(p.rvector2, ia, normalized(cross(getv(p.rvector, ia), d)));
          }
        }
      }
      if (nbond == 2) {
        if ((T[i1] == hydrogen || T[i2] == hydrogen) && T[i1] != T[i2] && p.disorderH) {
          // the second test reads i1 where i2 is meant (BondVectors.cpp:238-241)
          if (T[i1] == carbon || T[i1] == aromCarbon) ib = i1;
          if (T[i2] == carbon || T[i1] == aromCarbon) ib = i2;
          p.disorder[ia] = 1;
          if (ib >= 0 && ib < N) setv(p.rvector, ia, normalized(sub(pos(p, ia), pos(p, ib))));
        } else {
          V3 r2 = normalized(sub(pos(p, i2), pos(p, i1)));
          setv(p.rvector2, ia, r2);
          double rdot = dot(sub(pos(p, ia), pos(p, i1)), r2);
          setv(p.rvector, ia, normalized(sub(pos(p, ia), add(mul(r2, rdot), pos(p, i1)))));
        }
      }
    } else if (p.hbond[ia] == A1) {
      int nbond = 0;
      for (int ib = from; ib <= to; ib++) {
        if (ib == ia) continue;
        double rd2 = mag2(sub(pos(p, ia), pos(p, ib)));
        bool isH = T[ib] == hydrogen || T[ib] == nonHBhydrogen;
        if ((rd2 < 2.89 && !isH) || (rd2 < 1.69 && isH)) {
          if (nbond == 2) { nbond = 3; i3 = ib; }
          if (nbond == 1) { nbond = 2; i2 = ib; }
          if (nbond == 0) { nbond = 1; i1 = ib; }
        }
      }
      if (nbond == 0) log.warn("Nitrogen atom found with no bonded atoms, atom serial number %d", ia);
      if (nbond == 1) setv(p.rvector, ia, normalized(sub(pos(p, ia), pos(p, i1))));
      if (nbond == 2) setv(p.rvector, ia, normalized(sub(pos(p, ia), divs(add(pos(p, i2), pos(p, i1)), 2))));
      if (nbond == 3)
        setv(p.rvector, ia, normalized(sub(pos(p, ia), divs(add(add(pos(p, i1), pos(p, i2)), pos(p, i3)), 3))));
    }
  }
}

}  // namespace

void precompute(Problem& p, ParamLib& lib, Log& log, double* phaseMs) {
  // A GPF "parameter_file" is read only now, after the GPF (main.cpp:170-171):
  // it can change coeff_desolv and it resets the receptor indices that the bond
  // vectors and the disordered-hydrogen test look up by type name.
  if (!p.parameterLibraryFilename.empty()) {
    try {
      lib.loadFile(p.parameterLibraryFilename.c_str());
    } catch (ExitProgram& e) {
      log.print("%s\n", e.msg.c_str());
      throw;
    }
  }
  const auto t0 = std::chrono::steady_clock::now();
  energyTables(p);
  desolvTable(p, lib.coeff_desolv);
  const auto t1 = std::chrono::steady_clock::now();
  bondVectors(p, lib, log);
  const auto t2 = std::chrono::steady_clock::now();
  p.hydrogen = lib.recIndexOf("HD");
  if (!p.distDepDiel && p.epsilon.empty()) p.epsilon.assign(kMaxDist, 0.0);
  if (phaseMs) {
    phaseMs[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    phaseMs[1] = std::chrono::duration<double, std::milli>(t2 - t1).count();
  }
}

// ---------------------------------------------------------------------------
// Writers (GridMap.cpp:127-212, Utils.cpp:40-84, autogrid.h:255-258)
// ---------------------------------------------------------------------------
double roundOutput(double a) { return fabs(a) < 0.0005 ? 0 : floor(a * 1000 + 0.5) * 0.001; }

std::string mapHeader(const Problem& p) {
  char buf[4096];
  snprintf(buf, sizeof buf,
           "GRID_PARAMETER_FILE %s\nGRID_DATA_FILE %s\nMACROMOLECULE %s\nSPACING %.3lf\nNELEMENTS %d %d %d\nCENTER %.3lf %.3lf %.3lf\n",
           p.gpfName.c_str(), p.fldFilename.c_str(), p.receptorFilename.c_str(), p.spacing, p.n[0] - 1, p.n[1] - 1,
           p.n[2] - 1, p.center[0], p.center[1], p.center[2]);
  return buf;
}

// "%.3f\n" of roundOutput(v), or "0\n" when that is zero, without printf: the
// rounded value is an integer number of thousandths.
size_t formatValues(const float* v, int64_t count, char* buf) {
  char* o = buf;
  for (int64_t i = 0; i < count; i++) {
    double a = (double)v[i];
    if (fabs(a) < 0.0005) { *o++ = '0'; *o++ = '\n'; continue; }
    double k = floor(a * 1000 + 0.5);
    if (k == 0) { *o++ = '0'; *o++ = '\n'; continue; }
    if (!(fabs(k) < 9.0e15)) {  // inf/nan or astronomically large: defer to printf
      o += sprintf(o, "%.3f\n", k * 0.001);
      continue;
    }
    long long q = (long long)k;
    if (q < 0) { *o++ = '-'; q = -q; }
    long long ip = q / 1000;
    int fp = (int)(q % 1000);
    char tmp[24];
    int n = 0;
    do { tmp[n++] = char('0' + ip % 10); ip /= 10; } while (ip);
    while (n) *o++ = tmp[--n];
    *o++ = '.';
    *o++ = char('0' + fp / 100);
    *o++ = char('0' + (fp / 10) % 10);
    *o++ = char('0' + fp % 10);
    *o++ = '\n';
  }
  return (size_t)(o - buf);
}

static void writeValuesFile(const std::string& fname, const std::string& header, const float* v, int64_t n,
                            Log& log) {
  FILE* f = fopen(fname.c_str(), "w");
  if (!f) log.fatal(-2, "Cannot open grid map \"%s\" for writing.", fname.c_str());
  if (fwrite(header.data(), header.size(), 1, f) != 1) log.fatal(-2, "Not enough disk space.");
  // Format in parallel chunks, write in order.
  unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const int64_t chunk = std::max<int64_t>(1 << 16, (n + nt - 1) / nt);
  const int64_t nchunks = (n + chunk - 1) / chunk;
  std::vector<std::vector<char>> bufs(nchunks);
  std::vector<size_t> lens(nchunks);
  std::vector<std::thread> th;
  for (int64_t c = 0; c < nchunks; c++) {
    th.emplace_back([&, c] {
      int64_t b = c * chunk, e = std::min(n, b + chunk);
      bufs[c].resize((size_t)(e - b) * 24 + 16);
      lens[c] = formatValues(v + b, e - b, bufs[c].data());
    });
  }
  for (auto& t : th) t.join();
  for (int64_t c = 0; c < nchunks; c++)
    if (lens[c] && fwrite(bufs[c].data(), lens[c], 1, f) != 1) log.fatal(-2, "Not enough disk space.");
  if (fclose(f) != 0) log.fatal(-2, "Not enough disk space.");
}

// Every map file of the set at once: the values of all maps are formatted in
// parallel chunks (uninitialised buffers), then the files are written in
// parallel, one thread per file.  Errors are collected and reported after
// the threads have joined, with the reference's messages.
void writeAllMaps(const Problem& p, Log& log) {
  const int nm = p.numMaps();
  const int nmaps = nm + 2;
  const int64_t n = p.numPoints;
  const unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  const int64_t chunk = std::max<int64_t>(1 << 16, (n + nt - 1) / nt);
  const int64_t nchunks = n ? (n + chunk - 1) / chunk : 0;
  struct Piece {
    std::unique_ptr<char[]> buf;
    size_t len = 0;
  };
  std::vector<Piece> pieces((size_t)nmaps * nchunks);
  std::vector<std::string> names(nmaps);
  for (int m = 0; m < nmaps; m++) names[m] = m < nm ? p.maps[m].filename : (m == nm ? p.elecFilename : p.desolvFilename);
  const std::string header = mapHeader(p);
  std::atomic<int64_t> next(0);
  auto format = [&] {
    for (int64_t task; (task = next.fetch_add(1)) < (int64_t)pieces.size();) {
      const int m = (int)(task / nchunks);
      if (names[m].empty()) continue;
      const int64_t c = task % nchunks, b = c * chunk, e = std::min(n, b + chunk);
      Piece& pc = pieces[(size_t)task];
      pc.buf.reset(new char[(size_t)(e - b) * 24 + 16]);
      pc.len = formatValues(p.mapData() + (size_t)m * n + b, e - b, pc.buf.get());
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; t++) th.emplace_back(format);
  for (auto& t : th) t.join();
  th.clear();
  std::vector<int> err(nmaps, 0);  // 1 cannot open, 2 short write
  for (int m = 0; m < nmaps; m++) {
    if (names[m].empty()) continue;
    th.emplace_back([&, m] {
      FILE* f = fopen(names[m].c_str(), "w");
      if (!f) { err[m] = 1; return; }
      bool ok = fwrite(header.data(), header.size(), 1, f) == 1;
      for (int64_t c = 0; ok && c < nchunks; c++) {
        const Piece& pc = pieces[(size_t)m * nchunks + c];
        if (pc.len) ok = fwrite(pc.buf.get(), pc.len, 1, f) == 1;
      }
      if (fclose(f) != 0) ok = false;
      if (!ok) err[m] = 2;
    });
  }
  for (auto& t : th) t.join();
  for (int m = 0; m < nmaps; m++) {
    if (err[m] == 1) log.fatal(-2, "Cannot open grid map \"%s\" for writing.", names[m].c_str());
    if (err[m] == 2) log.fatal(-2, "Not enough disk space.");
  }
}

void writeMap(const Problem& p, int mapIndex, Log& log) {
  const int nm = p.numMaps();
  std::string fname = mapIndex < nm ? p.maps[mapIndex].filename : (mapIndex == nm ? p.elecFilename : p.desolvFilename);
  if (fname.empty()) return;
  writeValuesFile(fname, mapHeader(p), p.mapData() + (size_t)mapIndex * p.numPoints, p.numPoints, log);
}

void writeFloatingGrid(const Problem& p, Log& log) {
  if (!p.hasFloatingGrid()) return;
  FILE* f = fopen(p.floatingGridFilename.c_str(), "w");
  if (!f) log.fatal(-2, "can't open grid map \"%s\" for writing.", p.floatingGridFilename.c_str());
  std::string h = mapHeader(p);
  fwrite(h.data(), h.size(), 1, f);
  for (int64_t j = 0; j < p.numPoints; j++) fprintf(f, "%.3f\n", p.floatingGrid[j]);
  fclose(f);
}

void writeFld(const Problem& p, const char* programName, Log& log) {
  FILE* f = fopen(p.fldFilename.c_str(), "w");
  if (!f) log.fatal(-2, "can't create grid dimensions data file %s", p.fldFilename.c_str());
  const int nm = p.numMaps();
  const int numMaps = nm + 2 + (p.hasFloatingGrid() ? 1 : 0);
  fprintf(f, "# AVS field file\n#\n");
  fprintf(f, "# AutoDock Atomic Affinity and Electrostatic Grids\n#\n");
  fprintf(f, "# Created by %s.\n#\n", programName);
  fprintf(f, "#SPACING %.3f\n", float(p.spacing));
  fprintf(f, "#NELEMENTS %d %d %d\n", p.n[0] - 1, p.n[1] - 1, p.n[2] - 1);
  fprintf(f, "#CENTER %.3lf %.3lf %.3lf\n", p.center[0], p.center[1], p.center[2]);
  fprintf(f, "#MACROMOLECULE %s\n", p.receptorFilename.c_str());
  fprintf(f, "#GRID_PARAMETER_FILE %s\n#\n", p.gpfName.c_str());
  fprintf(f, "ndim=3\t\t\t# number of dimensions in the field\n");
  fprintf(f, "dim1=%d\t\t\t# number of x-elements\n", p.n[0]);
  fprintf(f, "dim2=%d\t\t\t# number of y-elements\n", p.n[1]);
  fprintf(f, "dim3=%d\t\t\t# number of z-elements\n", p.n[2]);
  fprintf(f, "nspace=3\t\t# number of physical coordinates per point\n");
  fprintf(f, "veclen=%d\t\t# number of affinity values at each point\n", numMaps);
  fprintf(f, "data=float\t\t# data type (byte, integer, float, double)\n");
  fprintf(f, "field=uniform\t\t# field type (uniform, rectilinear, irregular)\n");
  for (int i = 0; i < 3; i++)
    fprintf(f, "coord %d file=%s filetype=ascii offset=%d\n", i + 1, p.xyzFilename.c_str(), i * 2);
  for (int i = 0; i < nm; i++) fprintf(f, "label=%s-affinity\t# component label for variable %d\n", p.maps[i].type, i + 1);
  fprintf(f, "label=Electrostatics\t# component label for variable %d\n", numMaps - 2);
  fprintf(f, "label=Desolvation\t# component label for variable %d\n", numMaps - 1);
  if (p.hasFloatingGrid()) fprintf(f, "label=Floating_Grid\t# component label for variable %d\n", numMaps);
  fprintf(f, "#\n# location of affinity grid files and how to read them\n#\n");
  for (int i = 0; i < nm; i++) fprintf(f, "variable %d file=%s filetype=ascii skip=6\n", i + 1, p.maps[i].filename.c_str());
  fprintf(f, "variable %d file=%s filetype=ascii skip=6\n", nm + 1, p.elecFilename.c_str());
  fprintf(f, "variable %d file=%s filetype=ascii skip=6\n", nm + 2, p.desolvFilename.c_str());
  if (p.hasFloatingGrid())
    fprintf(f, "variable %d file=%s filetype=ascii skip=6\n", numMaps, p.floatingGridFilename.c_str());
  fclose(f);
}

}  // namespace ag
