// remc_replica.cpp - the Replica/Molecule facade over the batched C ABI.
// Host arithmetic (moves, centres, parsing) follows the reference's operation
// order in FP32/FP64 without contraction; every energy and every Metropolis
// step runs on the GPU through remc_b200.h.
#include "remc_replica.h"

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <utility>

namespace remc {

namespace {

void check(int rc, const char* what) {
  if (rc != REMC_OK) throw Error(std::string(what) + ": " + remc_last_error_string());
}

// Leading decimal number of s as sscanf("%f") reads it (0 when none).
float scan_float(const std::string& s) { return std::strtof(s.c_str(), nullptr); }
double scan_double(const std::string& s) { return std::strtod(s.c_str(), nullptr); }

std::string field(const std::string& s, size_t begin, size_t end) {
  if (begin >= s.size()) return std::string();
  return s.substr(begin, std::min(end, s.size()) - begin);
}

std::string first_token(const std::string& s) {
  std::istringstream is(s);
  std::string t;
  is >> t;
  return t;
}

std::vector<std::string> read_lines(const char* path, bool* ok) {
  std::ifstream in(path, std::ios::binary);
  std::vector<std::string> lines;
  *ok = bool(in);
  if (!in) return lines;
  std::string all((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  size_t p = 0;
  while (true) {
    size_t q = all.find('\n', p);
    std::string ln = all.substr(p, q == std::string::npos ? std::string::npos : q - p);
    if (!ln.empty() && ln.back() == '\r') ln.pop_back();
    lines.push_back(ln);
    if (q == std::string::npos) break;
    p = q + 1;
  }
  return lines;  // a trailing newline leaves one final empty line, as getline reads it
}

std::atomic<uint64_t> g_replica_serial{0};

}  // namespace

// ------------------------------------------------------------------ vectors
void Vector3double::normalizeInPlace() {
  const double m = std::sqrt(x * x + y * y + z * z);
  x /= m;
  y /= m;
  z /= m;
}

void Quaternion::normalize() {
  const double m = std::sqrt(w * w + x * x + y * y + z * z);
  w /= m;
  x /= m;
  y /= m;
  z /= m;
}

Quaternion Quaternion::operator*(const Quaternion& q) const {
  return Quaternion(w * q.w - x * q.x - y * q.y - z * q.z, w * q.x + x * q.w + y * q.z - z * q.y,
                    w * q.y - x * q.z + y * q.w + z * q.x, w * q.z + x * q.y - y * q.x + z * q.w);
}

Vector3f Quaternion::rotateVector(const Vector3f& v) const {
  const double w2 = w * w, x2 = x * x, y2 = y * y, z2 = z * z;
  const double wx = w * x, wy = w * y, wz = w * z, xy = x * y, xz = x * z, yz = y * z;
  const double vx = v.x, vy = v.y, vz = v.z;
  return Vector3f(float(vx * (w2 + x2 - y2 - z2) + (vy * (xy - wz) + vz * (wy + xz)) * 2.0),
                  float((vx * (wz + xy) + vz * (yz - wx)) * 2.0 + vy * (w2 - x2 + y2 - z2)),
                  float((vx * (xz - wy) + vy * (yz + wx)) * 2.0 + vz * (w2 - x2 - y2 + z2)));
}

// ------------------------------------------------------------------ AminoAcids
bool AminoAcids::loadAminoAcidData(const char* path) {
  bool ok;
  const std::vector<std::string> lines = read_lines(path, &ok);
  if (!ok) return false;
  int n = 0;
  size_t i = 0;
  while (i < lines.size() && n < REMC_NUM_AMINO) {
    const std::string& ln = lines[i];
    if (ln.empty() || ln[0] == '#') {
      ++i;
      continue;
    }
    if (i + 4 >= lines.size()) return false;
    AminoAcid& a = data[n++];
    a.name = ln.substr(0, 19);
    a.sname = lines[i + 1].substr(0, 3);
    a.symbol = lines[i + 2].empty() ? 0 : lines[i + 2][0];
    a.vdwRadius = float(scan_double(lines[i + 3]));  // atof into a float member
    a.electrostaticCharge = scan_float(lines[i + 4]);
    i += 5;
  }
  return n == REMC_NUM_AMINO;
}

// 3-letter names match with the first letter upper and the rest lower case,
// 1-letter names match the symbol, longer names the full name (last match
// wins, as the reference scans downwards).
int AminoAcids::getAminoAcidIndex(const char* name) const {
  const std::string s(name ? name : "");
  if (s.empty()) return -1;
  std::string key = s;
  if (s.size() == 3) {
    key = std::string(1, char(std::toupper((unsigned char)s[0]))) +
          char(std::tolower((unsigned char)s[1])) + char(std::tolower((unsigned char)s[2]));
    for (int i = REMC_NUM_AMINO - 1; i >= 0; --i)
      if (data[i].sname == key) return i;
  } else if (s.size() == 1) {
    const char c = char(std::toupper((unsigned char)s[0]));
    for (int i = REMC_NUM_AMINO - 1; i >= 0; --i)
      if (data[i].symbol == c) return i;
  } else {
    key[0] = char(std::toupper((unsigned char)key[0]));
    for (int i = REMC_NUM_AMINO - 1; i >= 0; --i)
      if (data[i].name == key) return i;
  }
  return -1;
}

bool AminoAcids::loadLJPotentialData(const char* path) {
  bool ok;
  const std::vector<std::string> lines = read_lines(path, &ok);
  if (!ok) return false;
  std::vector<int> labels;
  int start = 0;
  for (const std::string& ln : lines) {
    if (ln.empty() || ln[0] == '#') continue;
    std::istringstream is(ln);
    std::vector<std::string> toks;
    for (std::string t; is >> t;) toks.push_back(t);
    if (labels.empty()) {
      for (const std::string& t : toks) labels.push_back(getAminoAcidIndex(t.c_str()));
      if (labels.size() != REMC_NUM_AMINO ||
          *std::min_element(labels.begin(), labels.end()) < 0)
        return false;
      continue;
    }
    if (start >= REMC_NUM_AMINO) break;
    if ((int)toks.size() - 1 < REMC_NUM_AMINO - start) return false;
    for (int j = start; j < REMC_NUM_AMINO; ++j) {
      const float v = scan_float(toks[1 + j - start]);
      LJpotentials[labels[start]][labels[j]] = v;
      LJpotentials[labels[j]][labels[start]] = v;
    }
    ++start;
  }
  return start == REMC_NUM_AMINO;
}

// ------------------------------------------------------------------ Molecule
// CA beads at fixed columns (atom name 13-16, residue 18-20, x/y/z 31-54). An
// empty line re-reads the previous one (the reference's line buffer is not
// cleared), so a final newline after an ATOM CA line repeats that bead.
// Centre = FP32 running sum / count; relative position = position - centre.
bool Molecule::initFromPDB(const char* pdbfilename) {
  bool ok;
  const std::vector<std::string> lines = read_lines(pdbfilename, &ok);
  if (!ok) return false;
  Residues.clear();
  std::string prev;
  for (std::string ln : lines) {
    if (ln.size() > 511) ln.resize(511);
    const std::string cur = ln.empty() ? prev : ln;
    if (!ln.empty()) prev = ln;
    size_t b = cur.find_first_not_of(' ');
    const std::string tok =
        b == std::string::npos ? std::string() : cur.substr(b, cur.find(' ', b) - b);
    if (tok != "ATOM") continue;
    if (first_token(field(cur, 12, 16)) != "CA") continue;
    const std::string res = first_token(field(cur, 17, 20));
    const int t = AminoAcidsData.getAminoAcidIndex(res.c_str());
    if (t < 0) throw Error(std::string(pdbfilename) + ": unknown residue name '" + res + "'");
    Residue r;
    r.position = Vector3f(scan_float(field(cur, 30, 38)), scan_float(field(cur, 38, 46)),
                          scan_float(field(cur, 46, 54)));
    r.aminoAcidIndex = t;
    r.electrostaticCharge = AminoAcidsData.data[t].electrostaticCharge;
    r.vdwRadius = AminoAcidsData.data[t].vdwRadius;
    Residues.push_back(r);
  }
  residueCount = (int)Residues.size();
  if (residueCount == 0) return false;
  float cx = 0.0f, cy = 0.0f, cz = 0.0f;
  for (const Residue& r : Residues) {
    cx += r.position.x;
    cy += r.position.y;
    cz += r.position.z;
  }
  const float n = float(residueCount);
  center = Vector3f(cx / n, cy / n, cz / n);
  position = center;
  for (Residue& r : Residues)
    r.relativePosition = Vector3f(r.position.x - center.x, r.position.y - center.y,
                                  r.position.z - center.z);
  filename = pdbfilename;
  return true;
}

bool Molecule::translate(const Vector3f& v) {
  center = Vector3f(center.x + v.x, center.y + v.y, center.z + v.z);
  position = Vector3f(position.x + v.x, position.y + v.y, position.z + v.z);
  for (Residue& r : Residues)
    r.position = Vector3f(r.position.x + v.x, r.position.y + v.y, r.position.z + v.z);
  return true;
}

void Molecule::setPosition(const Vector3f& v) {
  center = v;
  position = v;
  for (Residue& r : Residues)
    r.position = Vector3f(r.relativePosition.x + center.x, r.relativePosition.y + center.y,
                          r.relativePosition.z + center.z);
}

bool Molecule::rotateQ(const Vector3double& axis, double angle) {
  const double sina = std::sin(angle / 2.0), cosa = std::cos(angle / 2.0);
  Quaternion q(cosa, sina * axis.x, sina * axis.y, sina * axis.z);
  setRotation(q);
  return true;
}

void Molecule::setRotation(Quaternion q) {
  q.normalize();
  rotation = q * rotation;
  for (Residue& r : Residues) {
    r.relativePosition = q.rotateVector(r.relativePosition);
    r.position = Vector3f(r.relativePosition.x + center.x, r.relativePosition.y + center.y,
                          r.relativePosition.z + center.z);
  }
}

void Molecule::saveBeforeStateChange(const Molecule* m) {
  Residues = m->Residues;
  residueCount = m->residueCount;
  center = m->center;
  position = m->position;
  rotation = m->rotation;
}

void Molecule::undoStateChange(const Molecule* m) {
  std::copy(m->Residues.begin(), m->Residues.begin() + residueCount, Residues.begin());
  center = m->center;
  position = m->position;
  rotation = m->rotation;
}

// ------------------------------------------------------------------ Replica
Replica::Replica() : seed_(0x5EED0000ull + g_replica_serial.fetch_add(1)) {
  remc_default_params(&params_);
}

Replica::~Replica() { FreeDevice(); }

Replica::Replica(const Replica& r) : Replica() { copy(r); }

Replica& Replica::operator=(const Replica& r) {
  if (this != &r) copy(r);
  return *this;
}

void Replica::copy(const Replica& r) {
  FreeDevice();
  aminoAcids = r.aminoAcids;
  molecules = r.molecules;
  moleculeCount = r.moleculeCount;
  residueCount = r.residueCount;
  maxMoleculeSize = r.maxMoleculeSize;
  nonCrowderCount = r.nonCrowderCount;
  boundingValue = r.boundingValue;
  temperature = r.temperature;
  label = r.label;
  potential = r.potential;
  translateStep = r.translateStep;
  rotateStep = r.rotateStep;
  blockSize = r.blockSize;
  params_ = r.params_;
  paramsSet_ = r.paramsSet_;
  ljOverride_ = r.ljOverride_;
  std::memcpy(lj_, r.lj_, sizeof(lj_));
  crowderRadius_ = r.crowderRadius_;
  translateOnlyCrowders_ = r.translateOnlyCrowders_;
}

int Replica::loadMolecule(const char* pdbfilename) {
  Molecule m;
  m.AminoAcidsData = aminoAcids;
  m.index = moleculeCount;
  if (!m.initFromPDB(pdbfilename)) throw Error(std::string("cannot read ") + pdbfilename);
  residueCount += m.residueCount;
  maxMoleculeSize = std::max(maxMoleculeSize, m.residueCount);
  molecules.push_back(std::move(m));
  return moleculeCount++;
}

int Replica::loadMolecule(const char* pdbfilename, Vector3f position, Vector3double rotationAxis,
                          double rotationAmount) {
  const int i = loadMolecule(pdbfilename);
  rotationAxis.normalizeInPlace();
  molecules[i].setPosition(position);
  molecules[i].rotateQ(rotationAxis, rotationAmount);
  return i;
}

void Replica::setLJpotentials(const float* ljp) {
  std::memcpy(lj_, ljp, sizeof(lj_));
  ljOverride_ = true;
  if (h_) ReplicaDataToDevice();
}

void Replica::setParams(const remc_params& p) {
  params_ = p;
  paramsSet_ = true;
  if (h_) check(remc_set_params(h_, &params_), "remc_set_params");
}

void Replica::topology(std::vector<int>& mol_start, std::vector<int>& role,
                       std::vector<int>& type) const {
  mol_start.assign(1, 0);
  role.clear();
  type.clear();
  for (const Molecule& m : molecules) {
    mol_start.push_back(mol_start.back() + m.residueCount);
    role.push_back(m.isCrowder() ? -1 : 0);
    for (const Residue& r : m.Residues) type.push_back(m.isCrowder() ? REMC_NUM_AMINO : r.aminoAcidIndex);
  }
}

void Replica::packState(float* pos, float* rel, float* centre, double* quat) const {
  size_t b = 0;
  for (size_t k = 0; k < molecules.size(); ++k) {
    const Molecule& m = molecules[k];
    for (const Residue& r : m.Residues) {
      pos[3 * b] = r.position.x;
      pos[3 * b + 1] = r.position.y;
      pos[3 * b + 2] = r.position.z;
      rel[3 * b] = r.relativePosition.x;
      rel[3 * b + 1] = r.relativePosition.y;
      rel[3 * b + 2] = r.relativePosition.z;
      ++b;
    }
    centre[3 * k] = m.center.x;
    centre[3 * k + 1] = m.center.y;
    centre[3 * k + 2] = m.center.z;
    quat[4 * k] = m.rotation.w;
    quat[4 * k + 1] = m.rotation.x;
    quat[4 * k + 2] = m.rotation.y;
    quat[4 * k + 3] = m.rotation.z;
  }
}

void Replica::unpackState(const float* pos, const float* rel, const float* centre,
                          const double* quat) {
  size_t b = 0;
  for (size_t k = 0; k < molecules.size(); ++k) {
    Molecule& m = molecules[k];
    for (Residue& r : m.Residues) {
      r.position = Vector3f(pos[3 * b], pos[3 * b + 1], pos[3 * b + 2]);
      r.relativePosition = Vector3f(rel[3 * b], rel[3 * b + 1], rel[3 * b + 2]);
      ++b;
    }
    m.center = Vector3f(centre[3 * k], centre[3 * k + 1], centre[3 * k + 2]);
    m.position = m.center;
    m.rotation = Quaternion(quat[4 * k], quat[4 * k + 1], quat[4 * k + 2], quat[4 * k + 3]);
  }
}

void Replica::typeTables(float* vdw, float* charge, float* rho) const {
  for (int t = 0; t < REMC_MAX_TYPES; ++t) vdw[t] = charge[t] = rho[t] = 0.0f;
  for (int t = 0; t < REMC_NUM_AMINO; ++t) {
    vdw[t] = aminoAcids.data[t].vdwRadius;
    charge[t] = aminoAcids.data[t].electrostaticCharge;
    rho[t] = aminoAcids.data[t].vdwRadius * 0.5f;
  }
  for (int t = REMC_NUM_AMINO; t < REMC_MAX_TYPES; ++t) rho[t] = crowderRadius_;
}

bool Replica::sameTopology(const Replica& r) const {
  if (molecules.size() != r.molecules.size() || boundingValue != r.boundingValue) return false;
  for (size_t k = 0; k < molecules.size(); ++k) {
    const Molecule &a = molecules[k], &b = r.molecules[k];
    if (a.residueCount != b.residueCount || a.isCrowder() != b.isCrowder()) return false;
    for (int i = 0; i < a.residueCount; ++i)
      if (a.Residues[i].aminoAcidIndex != b.Residues[i].aminoAcidIndex) return false;
  }
  return true;
}

void Replica::ensureHandle() {
  std::vector<int> ms, role, type;
  topology(ms, role, type);
  if (h_ && ms == devMolStart_ && devBox_ == boundingValue) return;
  FreeDevice();
  if (molecules.empty()) throw Error("replica has no molecules");
  remc_system_desc d;
  d.n_beads = (int)type.size();
  d.n_mol = (int)molecules.size();
  d.n_replicas = 1;
  d.mol_start = ms.data();
  d.mol_role = role.data();
  d.bead_type = type.data();
  d.box = boundingValue;
  d.translate_only_crowders = translateOnlyCrowders_ ? 1 : 0;
  check(remc_create(&d, 1, &params_, &h_), "remc_create");
  devMolStart_ = ms;
  devBox_ = boundingValue;
  nonCrowderCount = 0;
  for (const Molecule& m : molecules) nonCrowderCount += m.isCrowder() ? 0 : 1;
}

void Replica::ReplicaDataToDevice() {
  ensureHandle();
  float vdw[REMC_MAX_TYPES], q[REMC_MAX_TYPES], rho[REMC_MAX_TYPES];
  typeTables(vdw, q, rho);
  check(remc_set_type_tables(h_, vdw, q, rho, ljOverride_ ? lj_ : &aminoAcids.LJpotentials[0][0]),
        "remc_set_type_tables");
  std::vector<float> pos(3 * residueCount), rel(3 * residueCount), cen(3 * molecules.size());
  std::vector<double> quat(4 * molecules.size());
  packState(pos.data(), rel.data(), cen.data(), quat.data());
  check(remc_upload_state(h_, pos.data(), rel.data(), cen.data(), quat.data()),
        "remc_upload_state");
  const double rs = rotateStep;
  check(remc_set_replica_params(h_, &temperature, &translateStep, &rs), "remc_set_replica_params");
  replicaIsOnDevice = true;
}

void Replica::ReplicaDataToHost() {
  if (!h_) throw Error("ReplicaDataToHost: replica is not on the device");
  std::vector<float> pos(3 * residueCount), rel(3 * residueCount), cen(3 * molecules.size());
  std::vector<double> quat(4 * molecules.size());
  check(remc_download_state(h_, pos.data(), rel.data(), cen.data(), quat.data()),
        "remc_download_state");
  unpackState(pos.data(), rel.data(), cen.data(), quat.data());
}

// The engine uploads whole replicas; a one-molecule update re-sends the state.
void Replica::MoleculeDataToDevice(int moleculeId) {
  if (moleculeId < 0 || moleculeId >= moleculeCount) throw Error("MoleculeDataToDevice: bad index");
  ReplicaDataToDevice();
}

void Replica::FreeDevice() {
  if (h_) remc_destroy(h_);
  h_ = nullptr;
  devMolStart_.clear();
  replicaIsOnDevice = false;
}

double Replica::E() {
  ReplicaDataToDevice();
  double e = 0.0;
  check(remc_energy_full(h_, &e), "remc_energy_full");
  return e;
}

double Replica::EonDevice() { return E(); }

// steps Metropolis steps of this replica on the GPU, starting from the energy
// of the current conformation; the state, potential and move counters are
// brought back to the host afterwards.
void Replica::MCSearch(int steps) {
  if (steps <= 0) return;
  ReplicaDataToDevice();
  check(remc_energy_full(h_, nullptr), "remc_energy_full");
  check(remc_reset_counters(h_), "remc_reset_counters");
  check(remc_sweep(h_, steps, seed_, step_), "remc_sweep");
  step_ += (uint32_t)steps;
  ReplicaDataToHost();
  check(remc_get_energies(h_, &potential), "remc_get_energies");
  int a = 0, aA = 0, r = 0;
  check(remc_get_counters(h_, &a, &aA, &r), "remc_get_counters");
  accept += a;
  acceptA += aA;
  reject += r;
}

void Replica::exchangeReplicas(Replica& r) {
  std::swap(label, r.label);
  std::swap(temperature, r.temperature);
  std::swap(totalAcceptReject, r.totalAcceptReject);
  std::swap(totalAccept, r.totalAccept);
  std::swap(boundSamples, r.boundSamples);
  std::swap(samplesSinceLastExchange, r.samplesSinceLastExchange);
  std::swap(totalBoundSamples, r.totalBoundSamples);
  std::swap(totalSamples, r.totalSamples);
}

// ------------------------------------------------------------------ ReplicaExchange
ReplicaExchange::ReplicaExchange(std::vector<Replica*> replicas, uint64_t seed)
    : reps_(std::move(replicas)), seed_(seed) {
  if (reps_.empty()) throw Error("ReplicaExchange: no replicas");
  for (size_t k = 1; k < reps_.size(); ++k) {
    if (!reps_[k]->sameTopology(*reps_[0]))
      throw Error("ReplicaExchange: replicas must share topology and box");
    if (!(reps_[k]->temperature > reps_[k - 1]->temperature))
      throw Error("ReplicaExchange: temperatures must increase strictly");
  }
  const Replica& r0 = *reps_[0];
  std::vector<int> ms, role, type;
  r0.topology(ms, role, type);
  remc_system_desc d;
  d.n_beads = (int)type.size();
  d.n_mol = (int)r0.molecules.size();
  d.n_replicas = (int)reps_.size();
  d.mol_start = ms.data();
  d.mol_role = role.data();
  d.bead_type = type.data();
  d.box = r0.boundingValue;
  d.translate_only_crowders = r0.translateOnlyCrowders_ ? 1 : 0;
  check(remc_create(&d, 1, &r0.params_, &h_), "remc_create");
  for (Replica* r : reps_) {
    ladder_.push_back(r->temperature);
    labelOfTemp_.push_back(r->label);
  }
  upload();
}

ReplicaExchange::~ReplicaExchange() {
  if (h_) remc_destroy(h_);
}

void ReplicaExchange::upload() {
  const Replica& r0 = *reps_[0];
  float vdw[REMC_MAX_TYPES], q[REMC_MAX_TYPES], rho[REMC_MAX_TYPES];
  r0.typeTables(vdw, q, rho);
  check(remc_set_type_tables(h_, vdw, q, rho,
                             r0.ljOverride_ ? r0.lj_ : &r0.aminoAcids.LJpotentials[0][0]),
        "remc_set_type_tables");
  const size_t R = reps_.size(), nb = 3 * (size_t)r0.residueCount, nm = r0.molecules.size();
  std::vector<float> pos(R * nb), rel(R * nb), cen(R * 3 * nm);
  std::vector<double> quat(R * 4 * nm);
  std::vector<float> ts(R);
  std::vector<double> rs(R);
  for (size_t k = 0; k < R; ++k) {
    reps_[k]->packState(&pos[k * nb], &rel[k * nb], &cen[k * 3 * nm], &quat[k * 4 * nm]);
    ts[k] = reps_[k]->translateStep;
    rs[k] = reps_[k]->rotateStep;
  }
  check(remc_upload_state(h_, pos.data(), rel.data(), cen.data(), quat.data()),
        "remc_upload_state");
  check(remc_set_replica_params(h_, ladder_.data(), ts.data(), rs.data()),
        "remc_set_replica_params");
  check(remc_energy_full(h_, nullptr), "remc_energy_full");
}

void ReplicaExchange::download() {
  const Replica& r0 = *reps_[0];
  const size_t R = reps_.size(), nb = 3 * (size_t)r0.residueCount, nm = r0.molecules.size();
  std::vector<float> pos(R * nb), rel(R * nb), cen(R * 3 * nm);
  std::vector<double> quat(R * 4 * nm), e(R);
  std::vector<int> tmap(R), a(R), aA(R), rj(R);
  check(remc_download_state(h_, pos.data(), rel.data(), cen.data(), quat.data()),
        "remc_download_state");
  check(remc_get_energies(h_, e.data()), "remc_get_energies");
  check(remc_get_temperature_map(h_, tmap.data()), "remc_get_temperature_map");
  check(remc_get_counters(h_, a.data(), aA.data(), rj.data()), "remc_get_counters");
  check(remc_reset_counters(h_), "remc_reset_counters");
  for (size_t k = 0; k < R; ++k) {
    Replica& r = *reps_[k];
    r.unpackState(&pos[k * nb], &rel[k * nb], &cen[k * 3 * nm], &quat[k * 4 * nm]);
    r.potential = e[k];
    r.temperature = ladder_[tmap[k]];
    r.label = labelOfTemp_[tmap[k]];
    r.accept += a[k];
    r.acceptA += aA[k];
    r.reject += rj[k];
  }
}

void ReplicaExchange::autotune(int probe_steps) {
  check(remc_autotune(h_, probe_steps, seed_ ^ 0x5eedull, nullptr, nullptr, nullptr),
        "remc_autotune");
}

void ReplicaExchange::setCluster(int ctas_per_replica) {
  check(remc_set_cluster(h_, ctas_per_replica), "remc_set_cluster");
}

void ReplicaExchange::run(int n_blocks, int steps_per_block) {
  if (n_blocks <= 0) return;
  check(remc_run(h_, n_blocks, steps_per_block, seed_, step_, round_), "remc_run");
  step_ += (uint32_t)(n_blocks * steps_per_block);
  round_ += (uint32_t)n_blocks;
  download();
}

}  // namespace remc
