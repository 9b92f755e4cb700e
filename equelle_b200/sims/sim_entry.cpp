// In-process entry point of a generated-style simulator built as a shared
// library (compiled with -DEQUELLE_NO_MAIN next to the simulator source).
//
//   int eqg_sim_main(int argc, char** argv, eqg_sim_report* report)
//
// runs the program exactly as its main() would, then fills `report` with the
// device-clock duration and counters of every Newton solve (from the
// runtime's solve records) and the runtime's totals.  Returns 0, or 1 with the exception
// text in report->error.
#include "equelle/EquelleRuntimeCPU.hpp"

#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <cstring>

void equelleGeneratedCode(equelle::EquelleRuntimeCPU& er);

extern "C" {

struct eqg_sim_report {
    int64_t solves;
    double solve_ms[4096];      // duration of solve k
    double gap_ms[4096];        // start of solve k to start of solve k+1
    eqg_solve_info info[4096];  // counters of solve k
    double total_ms;            // first solve start to last solve end
    eqg_stats stats;
    char error[512];
    char profile[16384];        // eqg_runtime_kernel_profile JSON
};

int eqg_sim_main(int argc, char** argv, eqg_sim_report* report)
{
    std::memset(report, 0, sizeof(*report));
    const bool trace = std::getenv("EQG_SIM_TRACE") != nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    auto note = [&](const char* what) {
        if (!trace) return;
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        std::fprintf(stderr, "eqg_sim_main: %9.1f ms  %s\n", ms, what);
        std::fflush(stderr);
    };
    try {
        note("parameters");
        Opm::ParameterGroup param(argc, argv, false);
        note("runtime");
        equelle::EquelleRuntimeCPU er(param);
        eqg_runtime* rt = er.handle();
        note("program");
        try {
            equelleGeneratedCode(er);
        } catch (const std::exception& e) {
            // keep the counters of a run that stopped early
            std::strncpy(report->error, e.what(), sizeof(report->error) - 1);
            eqg_runtime_stats(rt, &report->stats);
            return 1;
        }
        note("report");
        equelle::detail::check(eqg_runtime_synchronize(rt));
        int64_t k = 0;
        int first_start = -1, last_end = -1, prev_start = -1;
        for (; k < 4096; ++k) {
            int s = 0, e = 0;
            if (eqg_runtime_solve_marks(rt, k, &s, &e) != EQG_OK) break;
            double ms = 0.0;
            equelle::detail::check(eqg_runtime_elapsed_ms(rt, s, e, &ms));
            report->solve_ms[k] = ms;
            equelle::detail::check(eqg_runtime_solve_info(rt, k, &report->info[k]));
            if (prev_start >= 0) {
                double g = 0.0;
                equelle::detail::check(eqg_runtime_elapsed_ms(rt, prev_start, s, &g));
                report->gap_ms[k - 1] = g;
            }
            if (first_start < 0) first_start = s;
            last_end = e;
            prev_start = s;
        }
        report->solves = k;
        if (first_start >= 0) equelle::detail::check(eqg_runtime_elapsed_ms(rt, first_start, last_end, &report->total_ms));
        if (k == 0 && !er.outputTags().empty()) {
            // an explicit program: its time steps are the intervals between
            // the outputs of the tag it outputs most often (the first such
            // tag; the end of output s to the start of output s + 1)
            std::string step_tag = er.outputTags().front();
            for (const auto& t : er.outputTags())
                if (er.outputMarks(t).size() > er.outputMarks(step_tag).size()) step_tag = t;
            const auto& marks = er.outputMarks(step_tag);
            int64_t steps = 0;
            for (size_t s = 0; s + 1 < marks.size() && s < 4096; ++s, ++steps) {
                double ms = 0.0;
                equelle::detail::check(eqg_runtime_elapsed_ms(rt, marks[s].second, marks[s + 1].first, &ms));
                report->solve_ms[s] = ms;
                if (s + 2 < marks.size()) {
                    equelle::detail::check(eqg_runtime_elapsed_ms(rt, marks[s].second, marks[s + 1].second, &ms));
                    report->gap_ms[s] = ms;
                }
            }
            report->solves = steps;
            if (steps > 0)
                equelle::detail::check(
                    eqg_runtime_elapsed_ms(rt, marks.front().second, marks[steps].first, &report->total_ms));
        }
        equelle::detail::check(eqg_runtime_stats(rt, &report->stats));
        int64_t need = 0;
        equelle::detail::check(eqg_runtime_kernel_profile(rt, report->profile, sizeof(report->profile), &need));
        note("done");
        return 0;
    } catch (const std::exception& e) {
        std::strncpy(report->error, e.what(), sizeof(report->error) - 1);
        return 1;
    }
}

}  // extern "C"
