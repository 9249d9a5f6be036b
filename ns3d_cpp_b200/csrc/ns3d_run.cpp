// time_advance (maincycle.cpp:7-112) with its monitor and output: host code
// over the library's C ABI.
//
// The reference synchronises with every step (it prints one line per step and
// tests its output schedule on the host). Here the loop runs on the device in
// segments: each ns3d_time_advance_segment call runs up to the next monitor
// step and ends early after a step whose if_output is set, so the host only
// waits where the reference writes something. What the reference writes there,
// and in which order, is reproduced:
//
//   every step: "Completed step n / max, Time = t / TotalTime" (verbose), from
//     the times the device recorded during the segment (ns3d_step_times)
//   monitor step (step == 1 or step % monitor_Stepfreq == 0):
//     compute_diagnostics           -> ns3d_residuals          (monitor_res)
//     compute_total_energy          -> ns3d_total_energy       (monitor_energy)
//     "[Step n] dt=..." on stdout                               (verbose)
//     write_residuals_tecplot       -> output/output_residuals.dat (monitor_res)
//     isotropic_post_process        -> spectrum file + statistics row (isotropic_analyse)
//   output step (if_output):
//     write_tecplot_field           -> output/time_<int(100000 t)>/field_rank0.dat
//                                                               (post_basicfield)
//     isotropic_post_process                                    (isotropic_analyse)
//
// The statistics row takes the spectrum as the reference does: rounded to the
// 6 digits of its spectrum file and read back (ana_isotropic.cpp:210-221).
//
// The reference's stdout switches to std::fixed with 6 decimals at its first
// "[Step" line and stays there, so the times of the lines printed before it
// (the first "Completed step" line) appear in the stream's default %g form.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <string>
#include <vector>

#include "ns3d_gpu.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Monitor {
    ns3d_ctx* ctx;
    ns3d_params p;
    std::string out;            // <workdir>/output
    double etot = 0.0;          // F.global_Etot: the last computed total energy
    double res[5] = {0, 0, 0, 0, 0};
    bool fixed = false;         // stdout in std::fixed, setprecision(6)

    // a time as the reference's stdout formats it at this point
    const char* fmt_time(double v, char* buf, size_t n) const {
        std::snprintf(buf, n, fixed ? "%.6f" : "%g", v);
        return buf;
    }

    // "Completed step" lines (maincycle.cpp:56-58) of the `done` steps ending
    // at step `last`
    ns3d_status completed(int last, int done, int max_steps) {
        std::vector<double> times(done);
        int got = 0;
        ns3d_status s = ns3d_step_times(ctx, times.data(), done, &got);
        if (s != NS3D_OK) return s;
        char a[64], b[64];
        for (int k = 0; k < std::min(got, done); ++k)
            std::printf("Completed step %d / %d, Time = %s / %s\n", last - done + 1 + k, max_steps,
                        fmt_time(times[k], a, sizeof a), fmt_time(p.TotalTime, b, sizeof b));
        return NS3D_OK;
    }

    // isotropic_post_process (postprocess.cpp:133-145) at time t
    ns3d_status isotropic(double t) {
        const int nbins = 2 * p.global_nx + 1;
        std::vector<double> Ek(nbins);
        ns3d_status s = ns3d_energy_spectrum(ctx, Ek.data(), nbins);
        if (s != NS3D_OK) return s;
        char name[96];
        std::snprintf(name, sizeof name, "/output_time_%.5f_spectrum.dat", t);
        if ((s = ns3d_spectrum_write((out + name).c_str(), Ek.data(), nbins)) != NS3D_OK) return s;
        // the values the reference reads back from that file
        for (double& e : Ek) {
            char txt[64];
            std::snprintf(txt, sizeof txt, "%g", e);
            e = std::strtod(txt, nullptr);
        }
        ns3d_turb_stats st;
        if ((s = ns3d_turbulence_stats_spectrum(ctx, Ek.data(), nbins, &st)) != NS3D_OK) return s;
        return ns3d_stats_write((out + "/turbulence_stats.dat").c_str(), t, &st);
    }

    ns3d_status monitor(int step, double t, double t_step, double t_elapsed, bool verbose) {
        ns3d_status s;
        if (p.monitor_res && (s = ns3d_residuals(ctx, res)) != NS3D_OK) return s;
        if (p.monitor_energy && (s = ns3d_total_energy(ctx, &etot)) != NS3D_OK) return s;
        if (verbose) {
            double dt = 0.0;
            if ((s = ns3d_last_dt(ctx, &dt)) != NS3D_OK) return s;
            std::printf("[Step %d] dt=%.6f  Time/step=%.6fs  Elapsed=%.6fs  Time=%.6f/%.6f", step,
                        dt, t_step, t_elapsed, t, p.TotalTime);
            if (p.monitor_energy) std::printf("  Ek_avg=%.6f", etot);
            std::printf("\n");
            std::fflush(stdout);
            fixed = true;
        }
        if (p.monitor_res &&
            (s = ns3d_residuals_write((out + "/output_residuals.dat").c_str(), step, res, etot)) !=
                NS3D_OK)
            return s;
        if (p.isotropic_analyse) return isotropic(t);
        return NS3D_OK;
    }

    ns3d_status output(double t) {
        ns3d_status s;
        if (p.post_basicfield) {
            const std::string dir = out + "/time_" + std::to_string(static_cast<int>(t * 100000));
            std::error_code ec;
            std::filesystem::create_directories(dir, ec);
            if ((s = ns3d_write_tecplot(ctx, (dir + "/field_rank0.dat").c_str(), t)) != NS3D_OK)
                return s;
        }
        if (p.isotropic_analyse) return isotropic(t);
        return NS3D_OK;
    }
};

// The first monitor step after `step` completed steps.
int next_monitor(int step, int freq) { return step == 0 ? 1 : (step / freq + 1) * freq; }

}  // namespace

extern "C" ns3d_status ns3d_run(ns3d_ctx* ctx, const char* workdir, int max_steps, int verbose,
                                double* time, int* steps_done) {
    if (!ctx || max_steps < 0) return NS3D_ERR_INVALID;
    Monitor m{ctx, {}, ""};
    ns3d_status s = ns3d_get_params(ctx, &m.p);
    if (s != NS3D_OK) return s;
    if (m.p.monitor_Stepfreq <= 0) return NS3D_ERR_INVALID;
    m.out = std::string(workdir && *workdir ? workdir : ".") + "/output";
    {
        std::error_code ec;
        std::filesystem::create_directories(m.out, ec);
    }
    const Clock::time_point t_start = Clock::now();
    Clock::time_point t_last = t_start;
    long long done0 = 0;
    if ((s = ns3d_completed_steps(ctx, &done0)) != NS3D_OK) return s;
    int step = (int)done0;  // a continued run numbers on (max_steps is the last step number)
    double t = 0.0;
    while (step < max_steps) {
        const int n = std::min(next_monitor(step, m.p.monitor_Stepfreq), max_steps) - step;
        int done = 0, events = 0;
        s = ns3d_time_advance_segment(ctx, n, &t, &done, &events);
        step += done;
        if (verbose && done > 0) {
            const ns3d_status sc = m.completed(step, done, max_steps);
            if (s == NS3D_OK) s = sc;
        }
        if (s != NS3D_OK || done == 0) break;
        if (step == 1 || step % m.p.monitor_Stepfreq == 0) {
            const Clock::time_point now = Clock::now();
            const double t_step = std::chrono::duration<double>(now - t_last).count();
            const double t_el = std::chrono::duration<double>(now - t_start).count();
            t_last = now;
            if ((s = m.monitor(step, t, t_step, t_el, verbose != 0)) != NS3D_OK) break;
        }
        if ((events & NS3D_EVENT_OUTPUT) && (s = m.output(t)) != NS3D_OK) break;
        if (events & NS3D_EVENT_END) break;
    }
    if (verbose) {
        char a[64];
        std::printf("Simulation complete. Total time: %s s\n",
                    m.fmt_time(std::chrono::duration<double>(Clock::now() - t_start).count(), a,
                               sizeof a));
        std::fflush(stdout);
    }
    if (time) *time = t;
    if (steps_done) *steps_done = step - (int)done0;
    return s;
}
