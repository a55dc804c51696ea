// K4: persistent batched RK8 tracker for charged particles in the electrostatic field of the
// charged elements (exact trajectory, B = 0).
//
// Reference path: KSRoot -> KSTrajTrajectoryExact::CalculateTrajectory -> KSMathRK8::Integrate
// (Kassiopeia/Math/Include/KSMathRK8.h:45-137, Butcher table :139-226) with the derivative of
// KSTrajTrajectoryExact::Differentiate + KSTrajTermPropagation::Differentiate
// (Kassiopeia/Trajectories/Source/KSTrajTrajectoryExact.cxx:302-316, KSTrajTermPropagation.cxx:25-35):
//   d/dt (t, s, x, p) = (1, |v|, v, q E(x)),  v = p / (m gamma),  gamma = sqrt(1 + p^2 / (m c)^2)
// with E(x) the Kahan-summed direct sum of KIntegratingFieldSolver::ElectricField.
//
// Layout: a CTA owns kTrackSlots slots (one per thread). Every RK stage of all slots of a CTA
// is one pass over the element records, streamed through a cyclic shared-memory ring
// (ElementRing, bulk copies; no CTA barrier per tile, so warps drift up to a tile apart); the
// 13 stage derivatives of each slot live in shared memory. A slot whose track ends (electrode
// hit, leaving the volume, step limit, non-finite state) or has taken `budget` steps in this
// launch writes it back and takes the next track index from a global work counter, so tracks
// of very different lengths keep every slot busy and one launch advances every listed track
// by at most `budget` steps; unfinished tracks stay active for the next launch.
#pragma once

#include "kemcu_kernels.cuh"

namespace kemcu
{

constexpr int kTrackSlots = 128;
constexpr int kStages = 13;
constexpr int kTrackPipe = 3;  // ring stages (the stage derivatives take most shared memory)
constexpr int kTrackK = 6;     // stored per stage and slot: v (3), q E (3)

// Butcher coefficients a[s][k] (row s gives stage value s from derivatives 0..s; row 12 is
// the final combination), the 13-stage eighth-order scheme of KSMathRK8.h:139-226
__constant__ double c_rk8[kStages][kStages];

inline void rk8_table(double a[kStages][kStages])
{
    for (int i = 0; i < kStages; i++)
        for (int j = 0; j < kStages; j++)
            a[i][j] = 0.;
    a[0][0] = 1. / 4.;
    a[1][0] = 5. / 72.; a[1][1] = 1. / 72.;
    a[2][0] = 1. / 32.; a[2][2] = 3. / 32.;
    a[3][0] = 106. / 125.; a[3][2] = -408. / 125.; a[3][3] = 352. / 125.;
    a[4][0] = 1. / 48.; a[4][3] = 8. / 33.; a[4][4] = 125. / 528.;
    a[5][0] = -1263. / 2401.; a[5][3] = 39936. / 26411.; a[5][4] = -64125. / 26411.; a[5][5] = 5520. / 2401.;
    a[6][0] = 37. / 392.; a[6][4] = 1625. / 9408.; a[6][5] = -2. / 15.; a[6][6] = 61. / 6720.;
    a[7][0] = 17176. / 25515.; a[7][3] = -47104. / 25515.; a[7][4] = 1325. / 504.; a[7][5] = -41792. / 25515.;
    a[7][6] = 20237. / 145800.; a[7][7] = 4312. / 6075.;
    a[8][0] = -23834. / 180075.; a[8][3] = -77824. / 1980825.; a[8][4] = -636635. / 633864.;
    a[8][5] = 254048. / 300125.; a[8][6] = -183. / 7000.; a[8][7] = 8. / 11.; a[8][8] = -324. / 3773.;
    a[9][0] = 12733. / 7600.; a[9][3] = -20032. / 5225.; a[9][4] = 456485. / 80256.; a[9][5] = -42599. / 7125.;
    a[9][6] = 339227. / 912000.; a[9][7] = -1029. / 4180.; a[9][8] = 1701. / 1408.; a[9][9] = 5145. / 2432.;
    a[10][0] = -27061. / 204120.; a[10][3] = 40448. / 280665.; a[10][4] = -1353775. / 1197504.;
    a[10][5] = 17662. / 25515.; a[10][6] = -71687. / 1166400.; a[10][7] = 98. / 225.; a[10][8] = 1. / 16.;
    a[10][9] = 3773. / 11664.;
    a[11][0] = 11203. / 8680.; a[11][3] = -38144. / 11935.; a[11][4] = 2354425. / 458304.;
    a[11][5] = -84046. / 16275.; a[11][6] = 673309. / 1636800.; a[11][7] = 4704. / 8525.; a[11][8] = 9477. / 10912.;
    a[11][9] = -1029. / 992.; a[11][11] = 729. / 341.;
    a[12][0] = 31. / 720.; a[12][5] = 16. / 75.; a[12][6] = 16807. / 79200.; a[12][7] = 16807. / 79200.;
    a[12][8] = 243. / 1760.; a[12][11] = 243. / 1760.; a[12][12] = 31. / 720.;
}

struct TrackParams
{
    double dt, charge, mass, c2;  // c2 = (speed of light)^2
    double hit_r2, max_r2;        // squared radii (0 disables)
    int max_steps, budget;
    int n_list;                   // number of track indices in list
    unsigned live;                // bit s: stage s's derivative has a nonzero weight somewhere
};

// Stages whose derivative no later stage and not the final combination uses (zero column of the
// Butcher table; stage 10 of this scheme: a[10][10] = a[11][10] = a[12][10] = 0). Their field
// sums cannot change the result, so the tracker does not evaluate them.
inline unsigned rk8_live_stages(const double a[kStages][kStages])
{
    unsigned live = 0u;
    for (int k = 0; k < kStages; k++)
        for (int r = k; r < kStages; r++)
            if (a[r][k] != 0.)
                live |= 1u << k;
    return live;
}

// state: n x 8; steps, status: n; list: n_list track indices to work on; next: work counter;
// done_steps: total steps taken (for statistics); dpsum (n, may be null): per track the sum over
// its steps of |p_after - p_before|, accumulated; flag |= 2 if a ring wait timed out.
// Dynamic shared memory: kStages * kTrackK * kTrackSlots doubles.
template<bool MIXED>
__global__ void __launch_bounds__(kTrackSlots) rk8_tracker_kernel(const double* __restrict__ rec, const double* __restrict__ sigma,
                                                                  int n_elem, double* __restrict__ state,
                                                                  int* __restrict__ steps, int* __restrict__ status,
                                                                  const int* __restrict__ list, unsigned* __restrict__ next,
                                                                  unsigned long long* __restrict__ done_steps,
                                                                  double* __restrict__ dpsum, TrackParams prm,
                                                                  int* __restrict__ flag)
{
    extern __shared__ __align__(16) double s_k[];  // [kStages][kTrackK][kTrackSlots]
    __shared__ __align__(128) RingStorage<1, kTrackPipe> S;
    __shared__ int s_abort;
    const int tid = threadIdx.x;
    auto K = [&](int st, int c) -> double& { return s_k[(st * kTrackK + c) * kTrackSlots + tid]; };
    if (tid == 0)
        s_abort = 0;
    ElementRing<1, kTrackPipe, true> R(S, 0, n_elem);  // synchronises the CTA
    auto side = [&](double (*sd)[kFieldTile], int t0, int cnt, int lane) {
        if (lane < cnt)
            sd[0][lane] = sigma[t0 + lane];
    };
    R.prologue(rec, side);
    const int ntiles = R.tiles();

    int track = -1, tsteps = 0;
    double y[8];
    double dps = 0.;
    int nstep = 0;
    auto pull = [&]() {
        track = -1;
        tsteps = 0;
        const unsigned w = atomicAdd(next, 1u);
        if (w < (unsigned) prm.n_list) {
            track = list[w];
            for (int c = 0; c < 8; c++)
                y[c] = state[(size_t) track * 8 + c];
            nstep = steps[track];
            dps = dpsum ? dpsum[track] : 0.;
        }
    };
    pull();
    unsigned long long my_steps = 0;
    int gi = 0;  // position in the ring's tile sequence
    bool ok = true;
    // every iteration is one RK8 step of all busy slots; ends when the list is exhausted (or a
    // ring wait of some warp timed out)
    while (true) {
        const int any = __syncthreads_or(track >= 0);
        if (!any || s_abort)
            break;
        double ds = 0.;  // sum over stages of a[12][k] |v_k|
        for (int st = 0; st < kStages; st++) {
            if (!((prm.live >> st) & 1u))
                continue;  // unused derivative (its column of the table is zero): not evaluated
            // stage position and momentum: value_{st-1} = y0 + dt sum_k a[st-1][k] k_k
            V3 X = v3(y[2], y[3], y[4]), Pm = v3(y[5], y[6], y[7]);
            if (track >= 0 && st > 0) {
                double sx = 0., sy = 0., sz = 0., px = 0., py = 0., pz = 0.;
                for (int k = 0; k < st; k++) {
                    if (!((prm.live >> k) & 1u))
                        continue;
                    const double a = c_rk8[st - 1][k];
                    sx += a * K(k, 0);
                    sy += a * K(k, 1);
                    sz += a * K(k, 2);
                    px += a * K(k, 3);
                    py += a * K(k, 4);
                    pz += a * K(k, 5);
                }
                X = v3(y[2] + prm.dt * sx, y[3] + prm.dt * sy, y[4] + prm.dt * sz);
                Pm = v3(y[5] + prm.dt * px, y[6] + prm.dt * py, y[7] + prm.dt * pz);
            }
            // E(X): one pass of all elements through the ring
            Kahan ex, ey, ez;
            if (ok) {
                for (int i = 0; i < ntiles; i++, gi++) {
                    if (!__all_sync(0xffffffffu, R.wait(gi))) {
                        ok = false;
                        s_abort = 1;
                        break;
                    }
                    if (track >= 0) {
                        const int cnt = R.count(gi);
                        for (int j = 0; j < cnt; j++) {
                            const Out4 r = epi<MIXED, false, true>(R.element(gi, j), X);
                            const double sg = R.side(gi, 0, j);
                            ex.add(r.ex * sg);
                            ey.add(r.ey * sg);
                            ez.add(r.ez * sg);
                        }
                    }
                    R.release(rec, gi, side);
                }
            }
            if (track >= 0) {
                const double p2 = dot(Pm, Pm);
                const double gam = sqrt(1. + p2 / (prm.mass * prm.mass * prm.c2));
                const double inv = 1. / (prm.mass * gam);
                const double vx = inv * Pm.x, vy = inv * Pm.y, vz = inv * Pm.z;
                K(st, 0) = vx;
                K(st, 1) = vy;
                K(st, 2) = vz;
                K(st, 3) = prm.charge * ex.s;
                K(st, 4) = prm.charge * ey.s;
                K(st, 5) = prm.charge * ez.s;
                ds += c_rk8[kStages - 1][st] * sqrt(vx * vx + vy * vy + vz * vz);
            }
        }
        if (track >= 0 && ok) {
            // final combination (row 12) for t (derivative 1), s (|v|), x and p
            double dtt = 0., d[6] = {0., 0., 0., 0., 0., 0.};
            for (int k = 0; k < kStages; k++) {
                const double a = c_rk8[kStages - 1][k];
                dtt += a;
                if (!((prm.live >> k) & 1u))
                    continue;
                for (int c = 0; c < 6; c++)
                    d[c] += a * K(k, c);
            }
            y[0] += prm.dt * dtt;
            y[1] += prm.dt * ds;
            double dp2 = 0.;
            for (int c = 0; c < 6; c++) {
                const double before = y[2 + c];
                y[2 + c] += prm.dt * d[c];
                if (c >= 3)
                    dp2 += (y[2 + c] - before) * (y[2 + c] - before);
            }
            dps += sqrt(dp2);  // KSStep::ContinuousMomentumChange (KSRootTrajectory.cxx:217-218)
            nstep++;
            my_steps++;
            const double r2 = y[2] * y[2] + y[3] * y[3] + y[4] * y[4];
            int stat = 0;
            bool finite = true;
            for (int c = 0; c < 8; c++)
                finite = finite && isfinite(y[c]);
            if (!finite)
                stat = 4;
            else if (prm.hit_r2 > 0. && r2 <= prm.hit_r2)
                stat = 1;
            else if (prm.max_r2 > 0. && r2 >= prm.max_r2)
                stat = 3;
            else if (nstep >= prm.max_steps)
                stat = 2;
            tsteps++;
            if (stat != 0 || tsteps >= prm.budget) {
                for (int c = 0; c < 8; c++)
                    state[(size_t) track * 8 + c] = y[c];
                steps[track] = nstep;
                if (dpsum)
                    dpsum[track] = dps;
                if (stat != 0)
                    status[track] = stat;
                pull();
            }
        }
    }
    R.finish(ok, flag);
    atomicAdd(done_steps, my_steps);
}

// list of ACTIVE tracks: list[atomicAdd(count)] = i for status[i] == 0
__global__ void active_list_kernel(const int* __restrict__ status, int n, int* __restrict__ list, unsigned* __restrict__ count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && status[i] == 0)
        list[atomicAdd(count, 1u)] = i;
}

}  // namespace kemcu
