// meso_b200: mesoBasic's driver with the GPU phase-field model.
//
//   meso_b200 [-i input.dat] [--print-params] [--timing] [Section/key=value ...]
//
// Reads the reference's input-parameter file (input.dat in the working
// directory unless -i names another), creates vtkoutput/ and removes old
// .vtk files there, builds every section marked "app = true" (only PFApp/
// exists, as in MesoBase.cpp), initialises it and writes step 0, then
// marches steps 1..Time/nstep writing output every nstep/numOutputs steps
// (MesoExecute.cpp:14-152).  numOutputs = 0 writes no output after step 0.
//
// --print-params prints the parameters the run would use, as JSON, and
// exits without touching the GPU.  --timing prints one JSON line with the
// wall time of the step loop at the end.
// Exit status: 0 on success, 1 on any error (message on stderr).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <exception>
#include <filesystem>
#include <memory>
#include <string>
#include <vector>

#include "chbasic_gpu.hpp"
#include "input_file.hpp"
#include "pf_model.hpp"

namespace fs = std::filesystem;

namespace {

std::string json_escape(const std::string& s)
{
    std::string o;
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o;
}

void print_params(const InputFile& in)
{
    std::printf("{\"sections\": [");
    const auto& secs = in.section_names();
    for (size_t i = 0; i < secs.size(); ++i) std::printf("%s\"%s\"", i ? ", " : "", json_escape(secs[i]).c_str());
    std::printf("], \"variables\": {");
    const auto& vars = in.variables();
    for (size_t i = 0; i < vars.size(); ++i)
        std::printf("%s\"%s\": \"%s\"", i ? ", " : "", json_escape(vars[i].first).c_str(),
                    json_escape(vars[i].second).c_str());
    std::printf("}, \"resolved\": {\"nx\": %d, \"ny\": %d, \"nz\": %d, \"dx\": %.17g, \"dy\": %.17g, \"dz\": %.17g, "
                "\"dt\": %.17g, \"nstep\": %d, \"numOutputs\": %d, \"iskip\": %d, \"jskip\": %d, \"kskip\": %d, "
                "\"type\": \"%s\", \"M\": %.17g, \"kap\": %.17g, \"co\": %.17g, \"noise_amp\": %.17g, "
                "\"seed\": %d, \"precision\": \"%s\"}}\n",
                in("Domain/nx", 1), in("Domain/ny", 1), in("Domain/nz", 1), in("Domain/dx", 1.0),
                in("Domain/dy", 1.0), in("Domain/dz", 1.0), in("Time/dt", 1.0), in("Time/nstep", 1),
                in("Output/numOutputs", 1), in("Output/iskip", 1), in("Output/jskip", 1), in("Output/kskip", 1),
                json_escape(in("PFApp/type", "CHBasic")).c_str(), in("PFApp/M", 1.0), in("PFApp/kap", 1.0),
                in("PFApp/co", 0.0), in("PFApp/noise_amp", 0.1), in("PFApp/seed", 42),
                json_escape(in("PFApp/precision", "fp64")).c_str());
}

int run(int argc, char** argv)
{
    std::string path = "input.dat";
    bool dry = false, timing = false;
    std::vector<std::pair<std::string, std::string>> overrides;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "-i" && i + 1 < argc) {
            path = argv[++i];
        } else if (a == "--print-params") {
            dry = true;
        } else if (a == "--timing") {
            timing = true;
        } else if (a.find('=') != std::string::npos && a[0] != '=') {
            overrides.emplace_back(a.substr(0, a.find('=')), a.substr(a.find('=') + 1));
        } else {
            std::fprintf(stderr, "meso_b200: unknown argument '%s'\n", a.c_str());
            return 1;
        }
    }
    InputFile in(path);
    for (const auto& kv : overrides) in.set(kv.first, kv.second);
    if (dry) {
        print_params(in);
        return 0;
    }

    const int nstep = in("Time/nstep", 0);
    const int numOutputs = in("Output/numOutputs", 1);
    int outInterval = numOutputs != 0 ? nstep / numOutputs : nstep + 1;
    // the reference divides by this interval inside the step loop (a crash
    // when it is 0); with no steps the loop never runs
    if (outInterval <= 0 && nstep > 0)
        throw std::invalid_argument("Output/numOutputs (" + std::to_string(numOutputs) + ") exceeds Time/nstep (" +
                                    std::to_string(nstep) + ")");

    // MesoExecute.cpp:28-31: fresh output directory
    fs::create_directories("vtkoutput");
    for (const auto& e : fs::directory_iterator("vtkoutput"))
        if (e.path().extension() == ".vtk") fs::remove(e.path());

    std::vector<std::unique_ptr<PFApp>> apps;
    for (const std::string& sec : in.section_names()) {
        if (in((sec + "app").c_str(), "false") != "true") continue;
        if (sec != "PFApp/") throw std::invalid_argument("section '" + sec + "' is not an application meso_b200 runs");
        apps.emplace_back(new PFApp(in));
    }
    for (auto& a : apps) {
        a->initSystem();
        a->writeOutput(0);
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (int step = 1; step < nstep + 1; ++step) {
        for (auto& a : apps) a->stepForward(step);
        if (step % outInterval == 0)
            for (auto& a : apps) a->writeOutput(step);
    }
    apps.clear();  // finishes the enqueued steps
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (timing) {
        const double sites = (double)in("Domain/nx", 1) * in("Domain/ny", 1) * in("Domain/nz", 1);
        std::printf("{\"steps\": %d, \"seconds\": %.6f, \"site_updates_per_s\": %.6e}\n", nstep, s,
                    s > 0 ? sites * nstep / s : 0.0);
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "meso_b200: %s\n", e.what());
        return 1;
    }
}
