// lgf_flow: command-line driver with the reference's positional arguments
// (LGF/LGF.cpp:30-31, ParseCLargs LGF.cpp:308-373) for the flow workflows:
//
//   lgf_flow NrDims extdofs beta shape[NrDims] cuts[NrDims] configStart configStop
//            flowSteps epsilon measureInterval dataFolder
//            [--workflow flow|resume=<t>|qdensity|measure] [--precision fp64|fp32mixed]
//            [--reunit-every k] [--device d] [--batch n]
//
// cuts are accepted and ignored (one GPU holds the whole lattice).  The
// workflow defaults to FlowSavedGaugeConfigurations; an integer in the epsilon
// position selects GenerateHeatBathGaugeConfigurations with ThermSteps =
// flowSteps, OR_per_HB = that integer and configSep = measureInterval, as in
// the reference's ParseCLargs.
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/lgf_b200.h"
#include "../../include/lgf_dropin.h"

int main(int argc, char** argv) {
    std::vector<std::string> pos;
    std::string workflow = "flow";
    int precision = LGF_PREC_FP64, reunit = 10, device = 0, batch = 0;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a.rfind("--workflow=", 0) == 0) workflow = a.substr(11);
        else if (a == "--workflow" && i + 1 < argc) workflow = argv[++i];
        else if (a.rfind("--precision=", 0) == 0) precision = a.substr(12) == "fp32mixed" ? LGF_PREC_FP32MIXED : LGF_PREC_FP64;
        else if (a == "--precision" && i + 1 < argc) precision = std::string(argv[++i]) == "fp32mixed" ? LGF_PREC_FP32MIXED : LGF_PREC_FP64;
        else if (a == "--reunit-every" && i + 1 < argc) reunit = std::atoi(argv[++i]);
        else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (a == "--batch" && i + 1 < argc) batch = std::atoi(argv[++i]);
        else pos.push_back(a);
    }
    if (pos.size() < 3) {
        std::cerr << "usage: lgf_flow NrDims extdofs beta shape[NrDims] cuts[NrDims] start stop steps eps interval folder\n";
        return 2;
    }
    const int NrDims = std::stoi(pos[0]);
    const int extdofs = std::stoi(pos[1]);
    const double beta = std::stod(pos[2]);
    if (pos.size() < (size_t)(3 + 2 * NrDims + 6)) {
        std::cerr << "lgf_flow: expected " << 3 + 2 * NrDims + 6 << " positional arguments\n";
        return 2;
    }
    std::vector<int> shape, cuts;
    size_t i = 3;
    for (int d = 0; d < NrDims; ++d) {
        shape.push_back(std::stoi(pos[i + d]));
        cuts.push_back(std::stoi(pos[i + NrDims + d]));
    }
    i += 2 * NrDims;
    const int start = std::stoi(pos[i++]);
    const int stop = std::stoi(pos[i++]);
    const int steps = std::stoi(pos[i++]);
    // an integer in the epsilon position selects the heatbath (ParseCLargs, LGF.cpp:326-335)
    const std::string eps_arg = pos[i++];
    size_t used = 0;
    std::stoi(eps_arg, &used);
    const bool heatbath = used == eps_arg.size();
    const double eps = heatbath ? 0.0 : std::stod(eps_arg);
    const int interval = std::stoi(pos[i++]);
    const std::string folder = pos[i++];
    if (heatbath && workflow == "flow") workflow = "heatbath";
    std::cout << "Started Parallel Session with 1 processes...\n";
    if (lgf_dropin_configure(precision, reunit, device) != LGF_OK ||
        (batch > 0 && lgf_dropin_set_batch(batch) != LGF_OK)) {
        std::cerr << "lgf_flow: bad engine options\n";
        return 2;
    }
    SimulationParameters params(NrDims, extdofs, shape, beta, cuts, "torus");
    FlowParameters flowParams(start, stop, steps, eps, interval, folder);
    if (workflow == "heatbath") {
        HBParameters hb(start, stop, steps, std::stoi(eps_arg), interval, folder);
        GenerateHeatBathGaugeConfigurations(params, hb);
    } else if (workflow == "flow") {
        FlowSavedGaugeConfigurations(params, flowParams);
    } else if (workflow.rfind("resume=", 0) == 0) {
        ResumeFlowedConfiguration(params, flowParams, std::stod(workflow.substr(7)));
    } else if (workflow == "qdensity") {
        MeasureQdensityDistribution(params, flowParams);
    } else if (workflow == "measure") {
        MeasureFlowedGaugeConfigurations(params, flowParams);
    } else {
        std::cerr << "lgf_flow: unknown workflow " << workflow << "\n";
        return 2;
    }
    return 0;
}
