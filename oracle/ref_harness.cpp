// Harness around the UNMODIFIED LGF reference sources (test infrastructure
// only; built by oracle/Makefile into oracle/_ref/lgf_ref).  It drives the
// reference's own entry points and member functions and prints/writes their
// results at full precision, so that the oracle restatement and the CUDA
// engine can be pinned against the reference itself.
//
// Subcommands (all single-rank through oracle/mpi_stub/mpi.h):
//   heatbath <folder> <beta> <N0> <N1> <N2> <N3> <therm> <OR_per_HB>
//       GenerateHeatBathGaugeConfigurations(params, HBParameters(0,0,therm,OR,1,folder))
//       (LGF/LGF.cpp:136-160); seed = $LGF_REF_SEED via oracle/seed_shim.h.
//   flow <folder> <beta> <N0> <N1> <N2> <N3> <start> <stop> <steps> <eps> <meas>
//       FlowSavedGaugeConfigurations(params, flowParams) (LGF/LGF.cpp:163-196)
//       with std::cout at 17 significant digits.
//   resume <folder> <beta> <N0> <N1> <N2> <N3> <start> <stop> <steps> <eps> <meas> <t_pickup>
//       ResumeFlowedConfiguration(params, flowParams, t_pickup) (LGF/LGF.cpp:197-226)
//       from <folder>'s saved <cfg>_Flowtime<t_pickup> file, std::cout as above.
//   qdensity|measureflowed <folder> <beta> <N0> <N1> <N2> <N3> <start> <stop> <steps> <eps> <meas>
//       MeasureQdensityDistribution / MeasureFlowedGaugeConfigurations
//       (LGF/LGF.cpp:113-123, :228-255) on the saved <cfg>_Flowtime<eps*steps> files.
//   kernels <links.bin> <N0> <N1> <N2> <N3> <out_prefix>
//       per-function outputs in global site order: staple (SU3_field.cpp:519),
//       flow gradient (Wilson.cpp:55), clover F (SU3_field.cpp:533),
//       improved F (SU3_field.cpp:588), per-site E and q terms
//       (EnergyDensity.cpp:13-20, TopologicalCharge.cpp:11-16) and the links
//       after one RK3 step (GradientFlow.cpp:22-60).
//   exp <in.bin> <out.bin>
//       HermTrLessExp (SU3_mat.cpp:216-289) on N matrices of 144 bytes.
//   cpubench <links.bin|hot> <N0> <N1> <N2> <N3> <steps> <meas_every>
//       the hot loop of FlowSavedGaugeConfigurations (LGF.cpp:166-188) without
//       file output, timed; prints one JSON line.
//   cpusplit <links.bin|hot> <N0> <N1> <N2> <N3> <steps>
//       the same objects, timed apart: each of <steps> GradientFlow::flow()
//       calls (no measurement falls due), then one GradientFlow::MakeMeasurements()
//       (Q then E, GradientFlow.cpp:76-83); prints one JSON line.
#include "LGF.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

void FlowSavedGaugeConfigurations(SimulationParameters& params, FlowParameters& flowParams);
void GenerateHeatBathGaugeConfigurations(SimulationParameters& params, HBParameters& HBparams);
void ResumeFlowedConfiguration(SimulationParameters& params, FlowParameters& flowParams, double flowTime_pickup);

namespace {

std::vector<int> shape_from(char** argv) {
    return {std::atoi(argv[0]), std::atoi(argv[1]), std::atoi(argv[2]), std::atoi(argv[3])};
}

// Mirrors SU3_field::loadSU3FromFile (SU3_field.cpp:329-340) for a raw path.
bool load_raw(SU3_field& U, Lattice& lat, const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    for (int site = U.Responsible_Start(); site < U.Responsible_Stop(); ++site) {
        for (int mu = 0; mu < 4; ++mu) {
            long long off = ((long long)lat.m_InternalToTotal_idx[site] * 4 + mu) * 144;
            std::fseek(f, off, SEEK_SET);
            if (std::fread(U(site, mu).getMemPointer(), 1, 144, f) != 144) {
                std::fclose(f);
                return false;
            }
        }
    }
    std::fclose(f);
    U.transfer_FieldValues();
    return true;
}

void put(std::vector<double>& out, size_t slot, su3_mat m) {
    for (int k = 0; k < 9; ++k) {
        out[slot * 18 + 2 * k] = m[k].Re;
        out[slot * 18 + 2 * k + 1] = m[k].Im;
    }
}

void write_file(const std::string& path, const std::vector<double>& v) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { std::perror(path.c_str()); std::exit(2); }
    std::fwrite(v.data(), sizeof(double), v.size(), f);
    std::fclose(f);
}

int cmd_kernels(int argc, char** argv) {
    if (argc < 7) return 2;
    std::string in = argv[1];
    std::vector<int> shape = shape_from(argv + 2);
    std::string prefix = argv[6];
    SimulationParameters params(4, 4, shape, 6.0, {0, 0, 0, 0}, "torus");
    Lattice lat(params, true);
    SU3_field U(lat, 4);
    if (!load_raw(U, lat, in)) { std::fprintf(stderr, "cannot read %s\n", in.c_str()); return 3; }
    const int V = lat.m_totalVolume;
    std::vector<double> staple((size_t)V * 4 * 18), grad((size_t)V * 4 * 18);
    std::vector<double> clov((size_t)V * 6 * 18), impr((size_t)V * 6 * 18);
    std::vector<double> edens(V), qdens(V);
    Wilson action(6.0);
    SU3_field Z(lat, 4);
    action.calculate_FlowGradient(U, Z);
    const int planes[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    for (int site = U.Responsible_Start(); site < U.Responsible_Stop(); ++site) {
        int g = lat.m_InternalToTotal_idx[site];
        for (int mu = 0; mu < 4; ++mu) {
            put(staple, (size_t)g * 4 + mu, U.staple(site, mu));
            put(grad, (size_t)g * 4 + mu, Z(site, mu));
        }
        for (int p = 0; p < 6; ++p) {
            put(clov, (size_t)g * 6 + p, U.FieldStrengthTensor(site, planes[p][0], planes[p][1]));
            put(impr, (size_t)g * 6 + p, U.Improved_fieldStrengthTensor(site, planes[p][0], planes[p][1]));
        }
        double e = 0.0;
        for (int mu = 0; mu < 4; mu++)
            for (int nu = mu + 1; nu < 4; nu++)
                e += (U.FieldStrengthTensor(site, mu, nu) * U.FieldStrengthTensor(site, mu, nu)).ReTr();
        double q = 0.0;
        q += (U.Improved_fieldStrengthTensor(site, 3, 2) * U.Improved_fieldStrengthTensor(site, 0, 1)).ReTr();
        q += (U.Improved_fieldStrengthTensor(site, 3, 1) * U.Improved_fieldStrengthTensor(site, 2, 0)).ReTr();
        q += (U.Improved_fieldStrengthTensor(site, 3, 0) * U.Improved_fieldStrengthTensor(site, 1, 2)).ReTr();
        edens[g] = e;
        qdens[g] = q;
    }
    write_file(prefix + "staple.bin", staple);
    write_file(prefix + "grad.bin", grad);
    write_file(prefix + "clover.bin", clov);
    write_file(prefix + "improved.bin", impr);
    write_file(prefix + "edens.bin", edens);
    write_file(prefix + "qdens.bin", qdens);
    // one RK3 step with no measurement (measEvery larger than 1 step)
    GradientFlow flowing(action, U, 0.01, 1000000);
    flowing.flow();
    std::vector<double> after((size_t)V * 4 * 18);
    for (int site = U.Responsible_Start(); site < U.Responsible_Stop(); ++site) {
        int g = lat.m_InternalToTotal_idx[site];
        for (int mu = 0; mu < 4; ++mu) put(after, (size_t)g * 4 + mu, U(site, mu));
    }
    write_file(prefix + "rk3step.bin", after);
    return 0;
}

int cmd_exp(int argc, char** argv) {
    if (argc < 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    std::vector<double> in;
    double buf[18];
    while (std::fread(buf, sizeof(double), 18, f) == 18) in.insert(in.end(), buf, buf + 18);
    std::fclose(f);
    size_t n = in.size() / 18;
    std::vector<double> out(in.size());
    for (size_t i = 0; i < n; ++i) {
        su3_mat m;
        for (int k = 0; k < 9; ++k) m[k] = C_double(in[i * 18 + 2 * k], in[i * 18 + 2 * k + 1]);
        put(out, i, HermTrLessExp(m));
    }
    write_file(argv[2], out);
    return 0;
}

int cmd_cpubench(int argc, char** argv) {
    if (argc < 8) return 2;
    std::string in = argv[1];
    std::vector<int> shape = shape_from(argv + 2);
    int steps = std::atoi(argv[6]);
    int meas = std::atoi(argv[7]);
    auto t0 = std::chrono::steady_clock::now();
    SimulationParameters params(4, 4, shape, 6.0, {0, 0, 0, 0}, "torus");
    Lattice lattice(params, true);
    Wilson action(params.getbeta());
    SU3_field U(lattice, params.getextdofs());
    if (in == "hot") {
        U.InitializeHotStart();
    } else if (!load_raw(U, lattice, in)) {
        std::fprintf(stderr, "cannot read %s\n", in.c_str());
        return 3;
    }
    auto t1 = std::chrono::steady_clock::now();
    // LGF.cpp:175-188, verbatim call sequence
    std::streambuf* saved = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    GradientFlow flowing(action, U, 0.01, meas);
    TopologicalCharge topCharge(U);
    flowing.Include_TopCharge(topCharge);
    EnergyDensity Edensity(U);
    flowing.Include_EnergyDensity(Edensity);
    auto t2 = std::chrono::steady_clock::now();
    // chunks of meas_every flow() calls; each chunk ends with the measurement
    // GradientFlow::flow makes itself (GradientFlow.cpp:56-58)
    std::vector<double> chunks;
    auto tc = t2;
    for (int i = 0; i < steps; i++) {
        flowing.flow();
        if ((i + 1) % meas == 0 || i + 1 == steps) {
            auto tn = std::chrono::steady_clock::now();
            chunks.push_back(std::chrono::duration<double>(tn - tc).count());
            tc = tn;
        }
    }
    auto t3 = std::chrono::steady_clock::now();
    std::cout.rdbuf(saved);
    double setup = std::chrono::duration<double>(t1 - t0).count();
    double flow = std::chrono::duration<double>(t3 - t2).count();
    long long V = (long long)shape[0] * shape[1] * shape[2] * shape[3];
    std::printf("{\"sites\": %lld, \"steps\": %d, \"meas_every\": %d, \"setup_s\": %.6f, \"flow_s\": %.6f, "
                "\"site_steps_per_s\": %.3f, \"chunks_s\": [",
                V, steps, meas, setup, flow, (double)V * steps / flow);
    for (size_t i = 0; i < chunks.size(); ++i) std::printf(i ? ", %.6f" : "%.6f", chunks[i]);
    std::printf("]}\n");
    return 0;
}

int cmd_cpusplit(int argc, char** argv) {
    if (argc < 7) return 2;
    std::string in = argv[1];
    std::vector<int> shape = shape_from(argv + 2);
    int steps = std::atoi(argv[6]);
    auto t0 = std::chrono::steady_clock::now();
    SimulationParameters params(4, 4, shape, 6.0, {0, 0, 0, 0}, "torus");
    Lattice lattice(params, true);
    Wilson action(params.getbeta());
    SU3_field U(lattice, params.getextdofs());
    if (in == "hot") {
        U.InitializeHotStart();
    } else if (!load_raw(U, lattice, in)) {
        std::fprintf(stderr, "cannot read %s\n", in.c_str());
        return 3;
    }
    auto t1 = std::chrono::steady_clock::now();
    std::streambuf* saved = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    // measurement interval beyond the step count: flow() never measures here
    GradientFlow flowing(action, U, 0.01, steps + 1);
    TopologicalCharge topCharge(U);
    flowing.Include_TopCharge(topCharge);
    EnergyDensity Edensity(U);
    flowing.Include_EnergyDensity(Edensity);
    std::vector<double> step_s;
    for (int i = 0; i < steps; i++) {
        auto a = std::chrono::steady_clock::now();
        flowing.flow();
        step_s.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count());
    }
    auto m0 = std::chrono::steady_clock::now();
    flowing.MakeMeasurements();
    const double meas_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - m0).count();
    std::cout.rdbuf(saved);
    long long V = (long long)shape[0] * shape[1] * shape[2] * shape[3];
    std::printf("{\"sites\": %lld, \"steps\": %d, \"setup_s\": %.6f, \"measure_s\": %.6f, \"step_s\": [", V, steps,
                std::chrono::duration<double>(t1 - t0).count(), meas_s);
    for (size_t i = 0; i < step_s.size(); ++i) std::printf(i ? ", %.6f" : "%.6f", step_s[i]);
    std::printf("]}\n");
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    mpiWrapper::begin_parallelSession(argc, argv);
    if (argc < 2) {
        std::fprintf(stderr, "usage: lgf_ref heatbath|flow|resume|qdensity|measureflowed|kernels|exp|cpubench ...\n");
        return 2;
    }
    std::string cmd = argv[1];
    int rc = 2;
    if (cmd == "heatbath" && argc >= 10) {
        std::vector<int> shape = shape_from(argv + 4);
        SimulationParameters params(4, 4, shape, std::stod(argv[3]), {0, 0, 0, 0}, "torus");
        HBParameters hb(0, 0, std::atoi(argv[8]), std::atoi(argv[9]), 1, argv[2]);
        GenerateHeatBathGaugeConfigurations(params, hb);
        rc = 0;
    } else if (cmd == "flow" && argc >= 13) {
        std::vector<int> shape = shape_from(argv + 4);
        SimulationParameters params(4, 4, shape, std::stod(argv[3]), {0, 0, 0, 0}, "torus");
        FlowParameters fp(std::atoi(argv[8]), std::atoi(argv[9]), std::atoi(argv[10]), std::stod(argv[11]),
                          std::atoi(argv[12]), argv[2]);
        std::cout << std::setprecision(17);
        FlowSavedGaugeConfigurations(params, fp);
        rc = 0;
    } else if (cmd == "resume" && argc >= 14) {
        // ResumeFlowedConfiguration (LGF.cpp:197-226) from the saved <cfg>_Flowtime<t> file
        std::vector<int> shape = shape_from(argv + 4);
        SimulationParameters params(4, 4, shape, std::stod(argv[3]), {0, 0, 0, 0}, "torus");
        FlowParameters fp(std::atoi(argv[8]), std::atoi(argv[9]), std::atoi(argv[10]), std::stod(argv[11]),
                          std::atoi(argv[12]), argv[2]);
        std::cout << std::setprecision(17);
        ResumeFlowedConfiguration(params, fp, std::stod(argv[13]));
        rc = 0;
    } else if ((cmd == "qdensity" || cmd == "measureflowed") && argc >= 13) {
        // MeasureQdensityDistribution (LGF.cpp:113-123) / MeasureFlowedGaugeConfigurations
        // (LGF.cpp:228-255) on <folder>'s saved <cfg>_Flowtime<eps*steps> files
        std::vector<int> shape = shape_from(argv + 4);
        SimulationParameters params(4, 4, shape, std::stod(argv[3]), {0, 0, 0, 0}, "torus");
        FlowParameters fp(std::atoi(argv[8]), std::atoi(argv[9]), std::atoi(argv[10]), std::stod(argv[11]),
                          std::atoi(argv[12]), argv[2]);
        std::cout << std::setprecision(17);
        if (cmd == "qdensity")
            MeasureQdensityDistribution(params, fp);
        else
            MeasureFlowedGaugeConfigurations(params, fp);
        rc = 0;
    } else if (cmd == "kernels") {
        rc = cmd_kernels(argc - 1, argv + 1);
    } else if (cmd == "exp") {
        rc = cmd_exp(argc - 1, argv + 1);
    } else if (cmd == "cpubench") {
        rc = cmd_cpubench(argc - 1, argv + 1);
    } else if (cmd == "cpusplit") {
        rc = cmd_cpusplit(argc - 1, argv + 1);
    }
    mpiWrapper::end_parallelSession();
    return rc;
}
