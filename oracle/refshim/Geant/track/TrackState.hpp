// Shim (oracle test infrastructure): the fields of the reference's TrackState
// (source/Geant/track/TrackState.hpp:30-232) that its EM models and processes
// touch, without the VecGeom navigation state.  The destructor records every
// TrackState a model builds and drops (the reference never pushes its
// secondaries), so the harness can read them back in construction order.
#pragma once
#include "Geant/core/Config.hpp"
#include "Geant/core/SystemOfUnits.hpp"
#include <cmath>
#include <vector>
namespace geantx {
struct ThreeVector {
  double v[3]{0, 0, 0};
  ThreeVector() {}
  ThreeVector(double a, double b, double c) { v[0] = a; v[1] = b; v[2] = c; }
  double &x() { return v[0]; }
  double &y() { return v[1]; }
  double &z() { return v[2]; }
  double x() const { return v[0]; }
  double y() const { return v[1]; }
  double z() const { return v[2]; }
  double Mag() const { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
  ThreeVector Unit() const { double m = Mag(); return m > 0 ? ThreeVector(v[0] / m, v[1] / m, v[2] / m) : *this; }
  ThreeVector operator-(const ThreeVector &o) const { return {v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]}; }
};
inline ThreeVector operator*(double s, const ThreeVector &a) { return {s * a.v[0], s * a.v[1], s * a.v[2]}; }
enum class TrackStatus : short { Alive, Killed, InFlight, Boundary, ExitingSetup, Physics, Postponed, New };
struct Element { double z; double GetZ() const { return z; } };
template <class T> using Vector_t = std::vector<T>;
struct MaterialProperties { const double *GetNumOfAtomsPerVolumeVect() const { return nullptr; } };
struct Material {
  Vector_t<Element *> e;
  const Vector_t<Element *> &GetElementVector() const { return e; }
  MaterialProperties *GetMaterialProperties() const { return nullptr; }
};
using Material_t = Material;
struct TrackPhysicsState {
  unsigned fParticleDefId = 0;
  double fEkin = 0, fMomentum = 0, fEdep = 0, fPstep = 0;
  unsigned fProcess = 0;
};
struct PhysicsProcessState { double fNumOfInteractLengthLeft = 0; double fPhysicsInteractLength = 0; };
struct TrackMaterialState { unsigned fMaterialId = 0; Material_t *fMaterial = nullptr; };
struct TrackSchedulingState { int fGVcode = 0; };
struct TrackState;
struct CapturedTrack { long seq; double ekin; double dir[3]; };
extern thread_local std::vector<CapturedTrack> *gxrefCapture;
extern thread_local long gxrefSeq;
struct TrackState {
  long fSeq = gxrefSeq++;
  bool fCapture = true;
  TrackStatus fStatus = TrackStatus::Alive;
  double fStep = 0, fTime = 0, fTotalLength = 0;
  ThreeVector fPos, fDir;
  TrackPhysicsState fPhysicsState;
  PhysicsProcessState fPhysicsProcessState[3];
  TrackMaterialState fMaterialState;
  TrackSchedulingState fSchedulingState;
  TrackState() = default;
  TrackState(const TrackState &) = default;
  TrackState &operator=(const TrackState &) = default;
  ~TrackState() {
    if (fCapture && gxrefCapture)
      gxrefCapture->push_back(CapturedTrack{fSeq, fPhysicsState.fEkin, {fDir.x(), fDir.y(), fDir.z()}});
  }
};
} // namespace geantx
