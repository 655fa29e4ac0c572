// Host-side model of one AutoGrid map-set job: the parsed GPF/PDBQT input, the
// parameter library, the precomputed lookup tables, the H-bond bond vectors and
// the output maps.  Everything here runs on the CPU before and after the GPU
// kernels; nothing here computes map values.
//
// The behaviour follows FastGrid (fastgrid_master/fastgrid/) so that a job that
// FastGrid accepts produces the same inputs to the map calculation:
//   InputDataLoader.cpp:100-797  (GPF + PDBQT), ParameterLibrary.cpp:34-234,
//   PairwiseInteractionEnergies.cpp:36-138, DesolvExpFunc.cpp:27-43,
//   BondVectors.cpp:45-393, GridMap.cpp:113-212, Utils.cpp:40-84.
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <stdexcept>

namespace ag {

// H-bonding character of an atom type (ParameterLibrary.h:29-37).
enum HBond { NON = 0, DS = 1, D1 = 2, AS = 3, A1 = 4, A2 = 5 };

constexpr int kMaxDist = 8192;        // table length, 0.01 A bins (autogrid.h:215)
constexpr int kNbCutoff = 8;          // non-bond cutoff in A (autogrid.h:216)
constexpr double kEintClamp = 100000.0;  // autocomm.h:98
constexpr int kMaxAtomTypes = 14;     // ligand map types (autocomm.h:102)
constexpr int kMaxMaps = 16;
constexpr int kNumAllTypes = 32;      // receptor types (autogrid.h:220)
constexpr double kApproxZero = 1.0e-6;
constexpr int kMaxGridPts = 1024;     // per axis (autocomm.h:94)
constexpr double kBig = 1.0e12;

// Thrown instead of exit(); carries the process exit code the reference uses
// (Exceptions.h; 911 missing GPF, -1 unknown type, -2 fatal error, 1 bad switch).
struct ExitProgram {
  int code;
  std::string msg;
};

struct AtomParam {
  char type[8] = {0};
  double Rij = 0, epsij = 0, vol = 0, solpar = 0, RijHB = 0, epsijHB = 0;
  int hbond = NON;
  int recIndex = -1, mapIndex = -1, bondIndex = 0;
};

// AD4 parameter library: FE coefficients + atom_par entries keyed by the first
// two characters of the type name (the reference hashes key[0] + 256*key[1]).
class ParamLib {
 public:
  double coeff_vdW = 0, coeff_hbond = 0, coeff_estat = 0, coeff_desolv = 0, coeff_tors = 0;
  explicit ParamLib(bool version4);
  void loadFile(const char* path);          // throws ExitProgram(-1) if missing
  void readLine(const char* line);
  AtomParam* find(const char* key);
  const AtomParam* find(const char* key) const;
  int recIndexOf(const char* key) const;

 private:
  static unsigned hashKey(const char* key);
  std::vector<int> slot_;                   // 65536 slots -> entries_ index or -1
  std::vector<AtomParam> entries_;
};

struct MapSpec {
  char type[4] = {0};
  std::string filename;
  bool isCovalent = false;
  bool isHBonder = false;
  int hbond = NON;
  double volProbe = 0, solparProbe = 0, Rij = 0, epsij = 0, RijHB = 0, epsijHB = 0;
  double nbpR[kNumAllTypes] = {0}, nbpEps[kNumAllTypes] = {0};
  int xA[kNumAllTypes] = {0}, xB[kNumAllTypes] = {0}, hbonder[kNumAllTypes] = {0};
};

// Simple .glg writer (the reference's LogFile); text parity is not a goal.
class Log {
 public:
  Log() = default;
  ~Log();
  void open(const char* path);              // empty -> stdout
  void print(const char* fmt, ...);
  void warn(const char* fmt, ...);          // also mirrored to stderr
  [[noreturn]] void fatal(int code, const char* fmt, ...);
  std::string programName = "fastgrid4";
 private:
  FILE* f_ = nullptr;
  bool own_ = false;
  int nWarn_ = 0;
};

struct Problem {
  // file names
  std::string gpfName;            // as given on the command line
  std::string fldFilename, xyzFilename, receptorFilename, floatingGridFilename, parameterLibraryFilename;
  std::string elecFilename, desolvFilename;

  // grid
  int n[3] = {0, 0, 0};           // points per axis (npts+1)
  int n2[3] = {0, 0, 0};          // npts/2
  int64_t numPoints = 0;
  double spacing = 0.375;
  double center[3] = {0, 0, 0};
  double cornerMin[3] = {0, 0, 0}, cornerMax[3] = {0, 0, 0};
  bool nptsSet = false;

  // receptor
  char receptorTypes[kNumAllTypes][3] = {{0}};
  int numReceptorTypes = 0;
  int numAtoms = 0;
  std::vector<double> charge, vol, solpar;
  std::vector<int> atomType, hbond;
  std::vector<double> xyzw;       // 4 per atom: centred x,y,z and the e-map weight
  std::vector<double> epsilon;    // 8192, 332/eps(r) (distance-dependent dielectric)

  double solparQ = 0.01097, invDielCal = 0, rSmooth = 0;
  double covHalfWidthSquaredInv = 1.0, covBarrier = 1000.0, covalentPoint[3] = {0, 0, 0};
  bool distDepDiel = false, disorderH = false;

  std::vector<MapSpec> maps;      // ligand (atom) maps
  bool mapsDeclared = false;

  // precomputed tables
  std::vector<double> energy;     // [numReceptorTypes][8192][numMaps]
  std::vector<double> sol;        // 8192, coeff_desolv * exp(-r^2 / (2*3.6^2)), sol[0] = 0
  int hydrogen = -1;              // receptor index of "HD" at map-calculation time

  // bond vectors (BondVectors.cpp)
  std::vector<uint8_t> disorder;
  std::vector<int> rexp;
  std::vector<double> rvector, rvector2;  // 3 per atom

  // outputs: [numMaps atom maps][e][d], x fastest, FP32, unrounded
  std::vector<float> out;
  const float* outView = nullptr;  // when set, the map set lives there (e.g. pinned memory) instead of `out`
  const float* mapData() const { return outView ? outView : out.data(); }
  std::vector<float> floatingGrid;

  int numMaps() const { return (int)maps.size(); }
  bool hasFloatingGrid() const { return !floatingGridFilename.empty(); }
};

// Load a GPF (and the PDBQT it names) exactly in the reference's order of
// operations.  Writes the .xyz file on the `gridcenter` line like the reference.
void loadGPF(Problem& p, ParamLib& lib, Log& log, const char* gpfPath);
// Tables, desolvation function, bond vectors (main.cpp:163-193 order).
// phaseMs (optional): [0] pair-energy and desolvation tables, [1] bond vectors, in ms.
void precompute(Problem& p, ParamLib& lib, Log& log, double* phaseMs = nullptr);

// Output
void writeFld(const Problem& p, const char* programName, Log& log);
void writeMap(const Problem& p, int mapIndex, Log& log);     // mapIndex in [0, numMaps+2)
void writeAllMaps(const Problem& p, Log& log);              // every map of the set, formatted and written in parallel
void writeFloatingGrid(const Problem& p, Log& log);
std::string mapHeader(const Problem& p);
double roundOutput(double a);
// Format `count` values (rounded like roundOutput) into `buf`; returns bytes.
size_t formatValues(const float* v, int64_t count, char* buf);

// 332/eps(r) of the Mehler-Solmajer dielectric (autogrid.h:233-239).
double distDepDielInv(double d);
}  // namespace ag

struct ag_synth_params;
namespace ag {
// Seeded synthetic receptor (synth.cpp): 3-decimal coordinates, type codes
// C OA N HD A SA = 0..5 and charges in thousandths.
int synthReceptor(const ag_synth_params* sp, std::vector<double>& xyz, std::vector<int>& type,
                  std::vector<long long>& milliCharge);
const char* synthTypeName(int t);

}  // namespace ag
