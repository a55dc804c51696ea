// kassiopeia_cuda.hh -- a KSRoot-level batch driver for Kassiopeia on the B200 backend
// (include/kemcu.h): many tracks of charged particles in an electrostatic boundary-element field
// advanced together by the device RK8 tracker, with the bookkeeping KSRoot::ExecuteTrack does
// per track (Kassiopeia/Simulation/Source/KSRoot.cxx:617-742).
//
// Reference path, per particle: KSRoot::ExecuteTrack -> ExecuteStep -> terminators (KSTermMaxSteps,
// KSTermMaxR, the navigator's surface hit, KSNavSpace.cxx:120-230) -> KSRootTrajectory with
// KSTrajTrajectoryExact (KSMathRK8.h:45-226, fixed time step KSTrajControlTime.cxx:14-18) ->
// the step's continuous time, length, energy and momentum changes added into KSTrack
// (KSRootTrajectory.cxx:208-221, KSRoot.cxx:689-705). Here:
//
//   * the initial particles (KSParticle) are packed into the exact trajectory's state
//     (t, s, x, p: KSTrajExactParticle.cxx:102-121) and advanced by kemcu_track_rk8 in launches of
//     at most StepsPerLaunch steps per track until every track has ended; particles of the same
//     charge and mass share the launches;
//   * a track ends after a step that brings it into the electrode (|x| <= electrode radius, the
//     analytic stand-in for the navigator's surface hit of the benchmark geometry; the step is not
//     truncated at the surface), that takes it out of the volume (|x| >= maximum radius,
//     KSTermMaxR), or after MaxSteps steps (KSTermMaxSteps: a track that reaches the limit ends
//     with TotalSteps = MaxSteps, as KSRoot does not count the terminating step);
//   * every KSTrack gets TrackId, TotalSteps, ContinuousTime, ContinuousLength,
//     ContinuousEnergyChange (kinetic, eV), ContinuousMomentumChange (sum over steps of |dp|,
//     accumulated on the device), zero discrete changes, InitialParticle, FinalParticle (state of
//     the last step, inactive) and TerminatorName.
//
// Header-only; include after the Kassiopeia headers (KSParticle.h, KSTrack.h) and link with
// -lkemcu. The device context must hold the geometry and charge densities (for instance the one
// of KEMField::KCUDAElectricFieldSolver::DeviceContainer()->Context()). Errors surface as
// std::runtime_error.
#pragma once

#include "KSParticle.h"
#include "KSTrack.h"
#include "kemcu.h"

#include <cmath>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace Kassiopeia
{

class KSCUDATrackBatch
{
  public:
    explicit KSCUDATrackBatch(kemcu_ctx* ctx) : fCtx(ctx)
    {
        if (!ctx)
            throw std::runtime_error("kemcu: KSCUDATrackBatch needs a device context");
    }
    // KSTrajControlTime: the fixed RK8 step in seconds
    void SetTime(double dt)
    {
        fTime = dt;
    }
    // KSTermMaxSteps
    void SetMaxSteps(int n, const std::string& name = "term_max_steps")
    {
        fMaxSteps = n;
        fMaxStepsName = name;
    }
    // electrode hit: |x| <= radius after a step (0 disables)
    void SetElectrode(double radius, const std::string& name = "electrode_hit")
    {
        fHit.sphere_radius = radius;
        fHitName = name;
    }
    // KSTermMaxR: |x| >= radius after a step (0 disables)
    void SetMaxR(double radius, const std::string& name = "term_max_r")
    {
        fHit.max_radius = radius;
        fMaxRName = name;
    }
    void SetStepsPerLaunch(int n)
    {
        fPerLaunch = n;
    }
    // KEMCU_FP64 (default) or KEMCU_MIXED arithmetic of the field sums
    void SetPrecision(int precision)
    {
        fPrecision = precision;
    }
    // device statistics of the last Execute, summed over its launches
    const kemcu_track_stats& LastStats() const
    {
        return fStats;
    }
    int LastLaunches() const
    {
        return fLaunches;
    }

    // KSRoot::ExecuteTrack for every particle of the batch; track i is particle i, with track id
    // first_track_id + i
    std::vector<KSTrack> Execute(const std::vector<KSParticle>& initial, int first_track_id = 0)
    {
        const size_t n = initial.size();
        std::vector<KSTrack> tracks(n);
        fStats = kemcu_track_stats{};
        fLaunches = 0;
        // particles of equal charge and mass run together
        std::map<std::pair<double, double>, std::vector<size_t>> groups;
        for (size_t i = 0; i < n; i++)
            groups[{initial[i].GetCharge(), initial[i].GetMass()}].push_back(i);
        for (auto& g : groups) {
            const std::vector<size_t>& idx = g.second;
            const size_t m = idx.size();
            std::vector<double> state(8 * m), dp(m, 0.);
            std::vector<int32_t> steps(m, 0), status(m, KEMCU_TRACK_ACTIVE);
            for (size_t k = 0; k < m; k++) {
                const KSParticle& p = initial[idx[k]];
                double* y = &state[8 * k];
                y[0] = p.GetTime();
                y[1] = p.GetLength();
                for (int c = 0; c < 3; c++) {
                    y[2 + c] = p.GetPosition()[c];
                    y[5 + c] = p.GetMomentum()[c];
                }
            }
            while (true) {
                kemcu_track_stats st{};
                const int rc = kemcu_track_rk8(fCtx, state.data(), steps.data(), status.data(), m, fTime, fMaxSteps,
                                               fPerLaunch, g.first.first, g.first.second, &fHit, fPrecision, &st,
                                               dp.data());
                if (rc != KEMCU_OK)
                    throw std::runtime_error(std::string("kemcu: ") + kemcu_last_error(fCtx));
                if (st.steps == 0)
                    break;
                fLaunches++;
                fStats.steps += st.steps;
                fStats.field_evals += st.field_evals;
                fStats.seconds += st.seconds;
                if (st.active == 0)
                    break;
            }
            for (size_t k = 0; k < m; k++) {
                const KSParticle& p0 = initial[idx[k]];
                const double* y = &state[8 * k];
                KSTrack& t = tracks[idx[k]];
                t.TrackId() = first_track_id + (int) idx[k];
                t.InitialParticle() = p0;
                KSParticle pf = p0;
                pf.SetTime(y[0]);
                pf.SetLength(y[1]);
                pf.SetPosition(y[2], y[3], y[4]);
                pf.SetMomentum(y[5], y[6], y[7]);
                pf.SetActive(false);
                t.FinalParticle() = pf;
                t.TotalSteps() = (unsigned int) steps[k];
                t.ContinuousTime() = pf.GetTime() - p0.GetTime();
                t.ContinuousLength() = pf.GetLength() - p0.GetLength();
                t.ContinuousEnergyChange() = pf.GetKineticEnergy_eV() - p0.GetKineticEnergy_eV();
                t.ContinuousMomentumChange() = dp[k];
                t.DiscreteEnergyChange() = 0.;
                t.DiscreteMomentumChange() = 0.;
                t.DiscreteSecondaries() = 0;
                t.NumberOfTurns() = 0;
                t.TerminatorName() = Terminator(status[k]);
                fStats.hit += status[k] == KEMCU_TRACK_HIT;
                fStats.max_steps += status[k] == KEMCU_TRACK_MAX_STEPS;
                fStats.left += status[k] == KEMCU_TRACK_LEFT;
                fStats.nonfinite += status[k] == KEMCU_TRACK_NONFINITE;
                fStats.active += status[k] == KEMCU_TRACK_ACTIVE;
            }
        }
        return tracks;
    }

  private:
    std::string Terminator(int status) const
    {
        switch (status) {
        case KEMCU_TRACK_HIT:
            return fHitName;
        case KEMCU_TRACK_MAX_STEPS:
            return fMaxStepsName;
        case KEMCU_TRACK_LEFT:
            return fMaxRName;
        case KEMCU_TRACK_NONFINITE:
            return "non_finite_state";
        default:
            return "";
        }
    }

    kemcu_ctx* fCtx;
    double fTime = 1e-11;
    int fMaxSteps = 10000;
    int fPerLaunch = 500;
    int fPrecision = KEMCU_FP64;
    kemcu_hit_model fHit{0., 0.};
    std::string fHitName = "electrode_hit", fMaxStepsName = "term_max_steps", fMaxRName = "term_max_r";
    kemcu_track_stats fStats{};
    int fLaunches = 0;
};

}  // namespace Kassiopeia
