// Host side of the drop-in: the reference's flow workflows on top of the C ABI.
//
// Keeps the reference's files and text output byte for byte:
//   input   <dataFolder>ensembles/su3/beta<b>/<N0>X<N1>X<N2>X<N3>/<method>/torus_extdof4_<id>.bin
//           V*4*144 bytes, global site order, no header (SU3_field.cpp:260-352)
//   output  <dataFolder>Observables/{Topological_Charge,EnergyDensity}/beta<b>/<shape>/GF/torus_extdof4_<id>.csv
//           "t,value\n" rows appended with default (6-digit) ostream formatting
//           (TopologicalCharge.cpp:31-71, EnergyDensity.cpp:37-80)
//           flowed links under method "GF", id "<cfg>_Flowtime<std::to_string(t)>" (LGF.cpp:194)
//   stdout  "Topological Charge = ..." / "Energy Density\t   = ..." per measurement,
//           Q before E (GradientFlow.cpp:77-84), and the load/save path lines.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <random>
#include <string>
#include <vector>

#include "../../include/lgf_b200.h"
#include "../../include/lgf_dropin.h"

namespace fs = std::filesystem;

namespace {

struct DropinState {
    lgf_ctx* ctx = nullptr;
    int precision = -1;
    int reunit_every = 10;
    int device = -1;
    int batch = -1;  // configurations flowed together by FlowSavedGaugeConfigurations (1 = one by one)
};
DropinState g_state;

int env_precision() {
    const char* p = std::getenv("LGF_PRECISION");
    if (p && (std::string(p) == "fp32mixed" || std::string(p) == "fp32" || std::string(p) == "1"))
        return LGF_PREC_FP32MIXED;
    return LGF_PREC_FP64;
}

lgf_ctx* context(int* rc) {
    if (g_state.precision < 0) g_state.precision = env_precision();
    if (g_state.device < 0) {
        const char* d = std::getenv("LGF_DEVICE");
        g_state.device = d ? std::atoi(d) : 0;
    }
    if (!g_state.ctx) {
        *rc = lgf_ctx_create(g_state.device, &g_state.ctx);
        if (*rc != LGF_OK) {
            std::cout << "LGF engine: cannot open CUDA device " << g_state.device << " (status " << *rc << ")\n";
            g_state.ctx = nullptr;
        }
    }
    return g_state.ctx;
}

std::string beta_string(double beta) {
    std::string s = std::to_string(beta);
    std::replace(s.begin(), s.end(), '.', '_');
    return s;
}

std::string shape_string(SimulationParameters& p) {
    std::string s;
    for (int i = 0; i < 3; ++i) s += std::to_string(p.getshape(i)) + "X";
    return s + std::to_string(p.getshape(3));
}

std::string ensemble_path(SimulationParameters& p, const std::string& method, const std::string& folder,
                          const std::string& id) {
    fs::path out(folder + "ensembles");
    out += "/su3/beta" + beta_string(p.getbeta()) + "/";
    out += shape_string(p) + "/" + method + "/";
    fs::create_directories(out);  // the reference creates the directory on load too (SU3_field.cpp:278)
    out += "torus_extdof4_" + id + ".bin";
    return out.string();
}

bool load_links(SimulationParameters& p, const std::string& method, const std::string& folder, const std::string& id,
                std::vector<double>& links) {
    const std::string path = ensemble_path(p, method, folder, id);
    std::cout << "Loading SU3 Field onto 1 processes\nFrom path " << path << "\n";
    std::cout.flush();
    std::FILE* f = std::fopen(path.c_str(), "rb");
    const size_t n = links.size();
    size_t got = 0;
    if (f) {
        got = std::fread(links.data(), sizeof(double), n, f);
        std::fclose(f);
    }
    if (got != n) {
        // The reference prints the MPI error and then blocks on std::cin
        // (SU3_field.cpp:300-309); the drop-in reports and skips the configuration.
        std::cout << LGF_EIO << " Error: cannot read " << n * sizeof(double) << " bytes from " << path << std::endl;
        return false;
    }
    std::cout << "File loaded \n";
    std::cout.flush();
    return true;
}

bool save_links(SimulationParameters& p, const std::string& method, const std::string& folder, const std::string& id,
                const std::vector<double>& links) {
    const std::string path = ensemble_path(p, method, folder, id);
    std::cout << "Saving SU3 Field to path " << path << "\n";
    std::cout.flush();
    std::FILE* f = std::fopen(path.c_str(), "r+b");
    if (!f) f = std::fopen(path.c_str(), "w+b");
    if (!f) {
        std::cout << LGF_EIO << " Error: cannot open " << path << std::endl;
        return false;
    }
    bool ok = std::fwrite(links.data(), sizeof(double), links.size(), f) == links.size();
    ok = (std::fclose(f) == 0) && ok;  // a failed flush is a failed save
    if (!ok) std::cout << LGF_EIO << " Error: cannot write " << path << std::endl;
    return ok;
}

void append_csv(SimulationParameters& p, const std::string& obs, const std::string& method, const std::string& folder,
                const std::string& id, const std::vector<double>& t, const std::vector<double>& v) {
    fs::path out(folder + "Observables");
    out += "/" + obs + "/beta" + beta_string(p.getbeta()) + "/";
    out += shape_string(p) + "/" + method + "/";
    fs::create_directories(out);
    out += "torus_extdof4" + id + ".csv";
    std::ofstream f(out.string(), std::ios_base::app);
    for (size_t i = 0; i < v.size(); ++i) f << t[i] << "," << v[i] << "\n";
}

bool check_params(SimulationParameters& p) {
    if (p.getNrDims() != 4 || p.getextdofs() != 4) {
        std::cout << "LGF engine: only NrDims = 4 and extdofs = 4 are supported\n";
        return false;
    }
    if (p.getLatticeType() != "torus") {
        std::cout << "LGF engine: lattice type " << p.getLatticeType() << " is not supported (use torus)\n";
        return false;
    }
    return true;
}

// Flow one configuration: upload, lgf_flow, print the measurements in the
// reference's order, download.  Returns the LGF status.
int flow_one(lgf_ctx* ctx, SimulationParameters& p, std::vector<double>& links, double eps, int steps, int meas,
             double t0, bool measure_t0, std::vector<double>& tv, std::vector<double>& Ev, std::vector<double>& Qv,
             double* t_end) {
    const int shape[4] = {p.getshape(0), p.getshape(1), p.getshape(2), p.getshape(3)};
    lgf_lattice* lat = nullptr;
    int rc = lgf_lattice_create(ctx, shape, g_state.precision, &lat);
    if (rc != LGF_OK) {
        std::cout << "LGF engine: " << lgf_last_error(ctx) << "\n";
        return rc;
    }
    rc = lgf_upload_links(lat, links.data());
    lgf_flow_opts o{};
    o.eps = eps;
    o.nsteps = steps;
    o.meas_every = meas;
    o.t0 = t0;
    o.measure_at_t0 = measure_t0 ? 1 : 0;
    o.reunit_every = g_state.precision == LGF_PREC_FP32MIXED ? g_state.reunit_every : 0;
    int nm = (measure_t0 ? 1 : 0) + (meas > 0 ? steps / meas : 0);
    tv.assign(std::max(nm, 1), 0.0);
    Ev.assign(std::max(nm, 1), 0.0);
    Qv.assign(std::max(nm, 1), 0.0);
    lgf_meas m{};
    m.capacity = nm;
    m.t = tv.data();
    m.E = Ev.data();
    m.Q = Qv.data();
    if (rc == LGF_OK) rc = lgf_flow(lat, &o, &m);
    if (rc == LGF_OK) rc = lgf_download_links(lat, links.data());
    if (rc != LGF_OK) std::cout << "LGF engine: " << lgf_last_error(ctx) << "\n";
    lgf_lattice_destroy(lat);
    tv.resize(nm);
    Ev.resize(nm);
    Qv.resize(nm);
    double t = t0;
    for (int s = 0; s < steps; ++s) t += eps;  // GradientFlow.cpp:52
    *t_end = t;
    if (rc == LGF_OK)
        for (int i = 0; i < nm; ++i) {
            std::cout << "Topological Charge = " << Qv[i] << "\n";
            std::cout.flush();
            std::cout << "Energy Density\t   = " << Ev[i] << "\n";
            std::cout.flush();
        }
    return rc;
}

}  // namespace

SimulationParameters::SimulationParameters(int NrDims, int extdofs, std::vector<int> shape, double beta,
                                           std::vector<int> cuts, std::string LatticeType) {
    m_NrDims = NrDims;
    m_extdofs = extdofs;
    m_shape = shape;
    m_beta = beta;
    m_cuts = cuts;
    m_LatticeType = LatticeType;
    if (m_LatticeType != "torus" && m_LatticeType != "torus_OpenT") {  // SimulationParameters.h:12-19
        std::cout << "Lattice type was not recognised!\n";
        std::cout << "Try <torus> or <torus_OpenT>" << std::endl;
        exit(EXIT_FAILURE);
    }
}

static int env_batch() {
    const char* b = std::getenv("LGF_BATCH");
    return b ? std::max(1, std::atoi(b)) : 1;
}

// FlowSavedGaugeConfigurations with up to g_state.batch configurations flowed
// together by lgf_batch_run (shared launches, one graph per RK3 step); each
// configuration's stdout lines, CSV rows and flowed file follow in the
// reference's order once its chunk is done.  The results are the same bits as
// flowing them one by one.
static int flow_saved_batched(SimulationParameters& params, FlowParameters& fp, lgf_ctx* ctx) {
    const std::string UpdateMethod = "LHMC_3_of_0_330000";  // LGF.cpp:164
    const long long V = 1LL * params.getshape(0) * params.getshape(1) * params.getshape(2) * params.getshape(3);
    const int shape[4] = {params.getshape(0), params.getshape(1), params.getshape(2), params.getshape(3)};
    const int steps = fp.getflowSteps(), meas = fp.getMeasuringInterval();
    const int nm = 1 + (meas > 0 ? steps / meas : 0);
    double flowTime = 0.0;
    for (int s = 0; s < steps; ++s) flowTime += fp.getepsilon();  // GradientFlow.cpp:52
    int status = LGF_OK;
    for (int c0 = fp.getConfigurationStart(); c0 <= fp.getConfigurationStop(); c0 += g_state.batch) {
        const int c1 = std::min(fp.getConfigurationStop(), c0 + g_state.batch - 1);
        struct Cfg {
            int id;
            std::vector<double> links, t, E, Q;
            lgf_meas m;
        };
        std::vector<Cfg> cfgs;
        cfgs.reserve(c1 - c0 + 1);
        for (int i = c0; i <= c1; ++i) {
            Cfg c;
            c.id = i;
            c.links.resize((size_t)V * 4 * 18);
            if (!load_links(params, UpdateMethod, fp.getdataFolder(), std::to_string(i), c.links)) {
                status = LGF_EIO;
                continue;
            }
            c.t.assign(nm, 0.0);
            c.E.assign(nm, 0.0);
            c.Q.assign(nm, 0.0);
            cfgs.push_back(std::move(c));
        }
        if (cfgs.empty()) continue;
        std::vector<lgf_job> jobs(cfgs.size());
        for (size_t k = 0; k < cfgs.size(); ++k) {
            Cfg& c = cfgs[k];
            c.m = lgf_meas{};
            c.m.capacity = nm;
            c.m.t = c.t.data();
            c.m.E = c.E.data();
            c.m.Q = c.Q.data();
            lgf_job& j = jobs[k];
            j = lgf_job{};
            std::memcpy(j.shape, shape, sizeof shape);
            j.precision = g_state.precision;
            j.links = c.links.data();
            j.flow.eps = fp.getepsilon();
            j.flow.nsteps = steps;
            j.flow.meas_every = meas;
            j.flow.t0 = 0.0;
            j.flow.measure_at_t0 = 1;
            j.flow.reunit_every = g_state.precision == LGF_PREC_FP32MIXED ? g_state.reunit_every : 0;
            j.meas = &c.m;
            j.links_out = c.links.data();  // read at admission, written at the end
        }
        const int rc = lgf_batch_run(ctx, jobs.data(), (int)jobs.size(), nullptr);
        if (rc != LGF_OK) {
            std::cout << "LGF engine: " << lgf_last_error(ctx) << "\n";
            status = rc;
            continue;
        }
        for (Cfg& c : cfgs) {
            for (int i = 0; i < nm; ++i) {
                std::cout << "Topological Charge = " << c.Q[i] << "\n";
                std::cout.flush();
                std::cout << "Energy Density\t   = " << c.E[i] << "\n";
                std::cout.flush();
            }
            const std::string ensembleNum = std::to_string(c.id);
            append_csv(params, "Topological_Charge", "GF", fp.getdataFolder(), "_" + ensembleNum, c.t, c.Q);
            append_csv(params, "EnergyDensity", "GF", fp.getdataFolder(), "_" + ensembleNum, c.t, c.E);
            if (!save_links(params, "GF", fp.getdataFolder(), ensembleNum + "_Flowtime" + std::to_string(flowTime),
                            c.links))
                status = LGF_EIO;
        }
    }
    return status;
}

static int flow_saved_impl(SimulationParameters& params, FlowParameters& fp) {
    if (!check_params(params)) return LGF_EINVAL;
    if (g_state.batch < 0) g_state.batch = env_batch();
    if (g_state.batch > 1) {
        int rc = LGF_OK;
        lgf_ctx* ctx = context(&rc);
        if (!ctx) return rc;
        const long long V = 1LL * params.getshape(0) * params.getshape(1) * params.getshape(2) * params.getshape(3);
        std::cout << "total Volume: " << V << std::endl;  // Lattice.cpp:199
        return flow_saved_batched(params, fp, ctx);
    }
    int rc = LGF_OK;
    lgf_ctx* ctx = nullptr;
    const std::string UpdateMethod = "LHMC_3_of_0_330000";  // LGF.cpp:164
    const long long V = 1LL * params.getshape(0) * params.getshape(1) * params.getshape(2) * params.getshape(3);
    std::cout << "total Volume: " << V << std::endl;  // Lattice.cpp:199
    int status = LGF_OK;
    for (int i = fp.getConfigurationStart(); i <= fp.getConfigurationStop(); i++) {
        std::vector<double> links((size_t)V * 4 * 18);
        const std::string ensembleNum = std::to_string(i);
        if (!load_links(params, UpdateMethod, fp.getdataFolder(), ensembleNum, links)) {
            status = LGF_EIO;
            continue;
        }
        if (!ctx && !(ctx = context(&rc))) return rc;
        std::vector<double> tv, Ev, Qv;
        double flowTime = 0.0;
        rc = flow_one(ctx, params, links, fp.getepsilon(), fp.getflowSteps(), fp.getMeasuringInterval(), 0.0, true,
                      tv, Ev, Qv, &flowTime);
        if (rc != LGF_OK) {
            status = rc;
            continue;
        }
        append_csv(params, "Topological_Charge", "GF", fp.getdataFolder(), "_" + ensembleNum, tv, Qv);
        append_csv(params, "EnergyDensity", "GF", fp.getdataFolder(), "_" + ensembleNum, tv, Ev);
        if (!save_links(params, "GF", fp.getdataFolder(), ensembleNum + "_Flowtime" + std::to_string(flowTime), links))
            status = LGF_EIO;
    }
    return status;
}

void FlowSavedGaugeConfigurations(SimulationParameters& params, FlowParameters& flowParams) {
    flow_saved_impl(params, flowParams);
}

static int resume_impl(SimulationParameters& params, FlowParameters& fp, double pickup) {
    if (!check_params(params)) return LGF_EINVAL;
    int rc = LGF_OK;
    lgf_ctx* ctx = nullptr;
    const long long V = 1LL * params.getshape(0) * params.getshape(1) * params.getshape(2) * params.getshape(3);
    int status = LGF_OK;
    for (int i = fp.getConfigurationStart(); i <= fp.getConfigurationStop(); i++) {  // LGF.cpp:201-225
        std::vector<double> links((size_t)V * 4 * 18);
        const std::string ensembleNum = std::to_string(i);
        if (!load_links(params, "GF", fp.getdataFolder(), ensembleNum + "_Flowtime" + std::to_string(pickup), links)) {
            status = LGF_EIO;
            continue;
        }
        if (!ctx && !(ctx = context(&rc))) return rc;
        std::vector<double> tv, Ev, Qv;
        double flowTime = pickup;
        rc = flow_one(ctx, params, links, fp.getepsilon(), fp.getflowSteps(), fp.getMeasuringInterval(), pickup, false,
                      tv, Ev, Qv, &flowTime);
        if (rc != LGF_OK) {
            status = rc;
            continue;
        }
        append_csv(params, "Topological_Charge", "GF", fp.getdataFolder(), "_" + ensembleNum, tv, Qv);
        append_csv(params, "EnergyDensity", "GF", fp.getdataFolder(), "_" + ensembleNum, tv, Ev);
        if (!save_links(params, "GF", fp.getdataFolder(), ensembleNum + "_Flowtime" + std::to_string(flowTime), links))
            status = LGF_EIO;
    }
    return status;
}

void ResumeFlowedConfiguration(SimulationParameters& params, FlowParameters& flowParams, double flowTime_pickup) {
    resume_impl(params, flowParams, flowTime_pickup);
}

static int qdensity_impl(SimulationParameters& params, FlowParameters& fp) {
    if (!check_params(params)) return LGF_EINVAL;
    int rc = LGF_OK;
    lgf_ctx* ctx = nullptr;
    const int shape[4] = {params.getshape(0), params.getshape(1), params.getshape(2), params.getshape(3)};
    const long long V = 1LL * shape[0] * shape[1] * shape[2] * shape[3];
    const double pickup = fp.getepsilon() * fp.getflowSteps();  // LGF.cpp:116
    const double PI = 4.0 * std::atan(1.0);
    const double PI2 = PI * PI;
    int status = LGF_OK;
    for (int i = fp.getConfigurationStart(); i <= fp.getConfigurationStop(); i++) {
        std::vector<double> links((size_t)V * 4 * 18);
        const std::string id = std::to_string(i) + "_Flowtime" + std::to_string(pickup);
        if (!load_links(params, "GF", fp.getdataFolder(), id, links)) {
            status = LGF_EIO;
            continue;
        }
        if (!ctx && !(ctx = context(&rc))) return rc;
        lgf_lattice* lat = nullptr;
        rc = lgf_lattice_create(ctx, shape, g_state.precision, &lat);
        std::vector<double> q((size_t)V);
        if (rc == LGF_OK) rc = lgf_upload_links(lat, links.data());
        if (rc == LGF_OK) rc = lgf_site_densities(lat, nullptr, q.data());
        if (lat) lgf_lattice_destroy(lat);
        if (rc != LGF_OK) {
            std::cout << "LGF engine: " << lgf_last_error(ctx) << "\n";
            status = rc;
            continue;
        }
        // the reference's prefactor (1.0/4.0*PI2) is pi^2/4 (QdensityDistribution.cpp:24), kept for
        // byte-compatible output
        for (auto& v : q) v = (1.0 / 4.0 * PI2) * v;
        fs::path out(fp.getdataFolder() + "Observables");
        out += "/Qdensity/beta" + beta_string(params.getbeta()) + "/";
        out += shape_string(params) + "/GF/";
        fs::create_directories(out);
        out += "torus_extdof1_" + id + ".bin";
        std::cout << "Saving Double Field to path " << out.string() << "\n";
        std::cout.flush();
        std::FILE* f = std::fopen(out.string().c_str(), "r+b");
        if (!f) f = std::fopen(out.string().c_str(), "w+b");
        if (!f || std::fwrite(q.data(), sizeof(double), q.size(), f) != q.size()) status = LGF_EIO;
        if (f && std::fclose(f) != 0) status = LGF_EIO;
    }
    return status;
}

void MeasureQdensityDistribution(SimulationParameters& params, FlowParameters& flowParams) {
    qdensity_impl(params, flowParams);
}

// MeasureFlowedGaugeConfigurations (LGF.cpp:228-255): the clover-F charge and
// the improved-F energy density of each flowed configuration, one CSV row each.
static int measure_flowed_impl(SimulationParameters& params, FlowParameters& fp) {
    if (!check_params(params)) return LGF_EINVAL;
    int rc = LGF_OK;
    lgf_ctx* ctx = nullptr;
    const int shape[4] = {params.getshape(0), params.getshape(1), params.getshape(2), params.getshape(3)};
    const long long V = 1LL * shape[0] * shape[1] * shape[2] * shape[3];
    const double pickup = fp.getepsilon() * fp.getflowSteps();  // LGF.cpp:231
    int status = LGF_OK;
    for (int i = fp.getConfigurationStart(); i <= fp.getConfigurationStop(); i++) {
        std::vector<double> links((size_t)V * 4 * 18);
        const std::string ensembleNum = std::to_string(i);
        if (!load_links(params, "GF", fp.getdataFolder(), ensembleNum + "_Flowtime" + std::to_string(pickup), links)) {
            status = LGF_EIO;
            continue;
        }
        if (!ctx && !(ctx = context(&rc))) return rc;
        lgf_lattice* lat = nullptr;
        double Eimp = 0.0, Qclov = 0.0;
        rc = lgf_lattice_create(ctx, shape, g_state.precision, &lat);
        if (rc == LGF_OK) rc = lgf_upload_links(lat, links.data());
        if (rc == LGF_OK) rc = lgf_measure_flowed(lat, &Eimp, &Qclov);
        if (lat) lgf_lattice_destroy(lat);
        if (rc != LGF_OK) {
            std::cout << "LGF engine: " << lgf_last_error(ctx) << "\n";
            status = rc;
            continue;
        }
        std::cout << "Topological Charge = " << Qclov << "\n";
        std::cout.flush();
        std::cout << "Energy Density\t   = " << Eimp << "\n";
        std::cout.flush();
        const std::vector<double> t{pickup};
        append_csv(params, "UnImprovedTopological_Charge", "GF", fp.getdataFolder(), "_" + ensembleNum, t, {Qclov});
        append_csv(params, "ImprovedEnergyDensity", "GF", fp.getdataFolder(), "_" + ensembleNum, t, {Eimp});
    }
    return status;
}

void MeasureFlowedGaugeConfigurations(SimulationParameters& params, FlowParameters& flowParams) {
    measure_flowed_impl(params, flowParams);
}

// GenerateHeatBathGaugeConfigurations (LGF.cpp:136-160): hot start and
// thermalisation for a new ensemble (ThermSteps != 0 and start == 0), else
// continue from the saved configuration `start`; then one saved configuration
// every configSep updates.  update(n) prints "step: i" per iteration like
// SU3_Heatbath::update (SU3_Heatbath.cpp:16-25).
static int heatbath_impl(SimulationParameters& params, HBParameters& hb, uint64_t seed) {
    if (!check_params(params)) return LGF_EINVAL;
    int rc = LGF_OK;
    lgf_ctx* ctx = context(&rc);
    if (!ctx) return rc;
    const int shape[4] = {params.getshape(0), params.getshape(1), params.getshape(2), params.getshape(3)};
    const long long V = 1LL * shape[0] * shape[1] * shape[2] * shape[3];
    const std::string method = "Heatbath_" + std::to_string(hb.getOR_per_HB()) + "_ORperHB";  // SU3_Heatbath.cpp:6
    lgf_lattice* lat = nullptr;
    rc = lgf_lattice_create(ctx, shape, g_state.precision, &lat);
    if (rc != LGF_OK) {
        std::cout << "LGF engine: " << lgf_last_error(ctx) << "\n";
        return rc;
    }
    std::vector<double> links((size_t)V * 4 * 18);
    const bool fresh = hb.getThermSteps() != 0 && hb.getConfigurationStart() == 0;
    if (fresh) {
        rc = lgf_hot_start(lat, seed);
    } else if (!load_links(params, method, hb.getdataFolder(), std::to_string(hb.getConfigurationStart()), links)) {
        rc = LGF_EIO;
    } else {
        rc = lgf_upload_links(lat, links.data());
    }
    auto update = [&](int n) {
        for (int i = 0; i < n && rc == LGF_OK; ++i) {
            rc = lgf_heatbath(lat, params.getbeta(), 1, hb.getOR_per_HB(), seed, nullptr);
            std::cout << "step: " << i << std::endl;
        }
    };
    auto save = [&](int cfg) {
        if (rc == LGF_OK) rc = lgf_download_links(lat, links.data());
        if (rc == LGF_OK && !save_links(params, method, hb.getdataFolder(), std::to_string(cfg), links)) rc = LGF_EIO;
    };
    if (fresh) {
        update(hb.getThermSteps());
        save(hb.getConfigurationStart());
    }
    for (int i = hb.getConfigurationStart() + 1; i <= hb.getConfigurationStop() && rc == LGF_OK; i++) {
        update(hb.getconfigSep());
        save(i);
    }
    if (rc != LGF_OK && rc != LGF_EIO) std::cout << "LGF engine: " << lgf_last_error(ctx) << "\n";
    lgf_lattice_destroy(lat);
    return rc;
}

static uint64_t env_seed() {
    const char* s = std::getenv("LGF_SEED");
    if (s) return std::strtoull(s, nullptr, 10);
    std::random_device rd;
    return ((uint64_t)rd() << 32) ^ rd();
}

void GenerateHeatBathGaugeConfigurations(SimulationParameters& params, HBParameters& HBparams) {
    heatbath_impl(params, HBparams, env_seed());
}

extern "C" {

int lgf_dropin_configure(int precision, int reunit_every, int device) {
    if (precision != LGF_PREC_FP64 && precision != LGF_PREC_FP32MIXED) return LGF_EINVAL;
    if (reunit_every < 0 || device < 0) return LGF_EINVAL;
    if (g_state.ctx && device != g_state.device) {
        lgf_ctx_destroy(g_state.ctx);
        g_state.ctx = nullptr;
    }
    g_state.precision = precision;
    g_state.reunit_every = reunit_every;
    g_state.device = device;
    return LGF_OK;
}

int lgf_dropin_set_batch(int configs) {
    if (configs < 1) return LGF_EINVAL;
    g_state.batch = configs;
    return LGF_OK;
}

int lgf_dropin_flow_saved(const int shape[4], double beta, int config_start, int config_stop, int flow_steps,
                          double epsilon, int measure_every, const char* data_folder) {
    if (!shape || !data_folder) return LGF_EINVAL;
    SimulationParameters p(4, 4, {shape[0], shape[1], shape[2], shape[3]}, beta, {0, 0, 0, 0}, "torus");
    FlowParameters f(config_start, config_stop, flow_steps, epsilon, measure_every, data_folder);
    return flow_saved_impl(p, f);
}

int lgf_dropin_resume_flowed(const int shape[4], double beta, int config_start, int config_stop, int flow_steps,
                             double epsilon, int measure_every, const char* data_folder, double flow_time_pickup) {
    if (!shape || !data_folder) return LGF_EINVAL;
    SimulationParameters p(4, 4, {shape[0], shape[1], shape[2], shape[3]}, beta, {0, 0, 0, 0}, "torus");
    FlowParameters f(config_start, config_stop, flow_steps, epsilon, measure_every, data_folder);
    return resume_impl(p, f, flow_time_pickup);
}

int lgf_dropin_measure_flowed(const int shape[4], double beta, int config_start, int config_stop, int flow_steps,
                              double epsilon, int measure_every, const char* data_folder) {
    if (!shape || !data_folder) return LGF_EINVAL;
    SimulationParameters p(4, 4, {shape[0], shape[1], shape[2], shape[3]}, beta, {0, 0, 0, 0}, "torus");
    FlowParameters f(config_start, config_stop, flow_steps, epsilon, measure_every, data_folder);
    return measure_flowed_impl(p, f);
}

int lgf_dropin_generate_heatbath(const int shape[4], double beta, int config_start, int config_stop, int therm_steps,
                                 int or_per_hb, int config_sep, const char* data_folder, uint64_t seed) {
    if (!shape || !data_folder || therm_steps < 0 || or_per_hb < 0 || config_sep < 0) return LGF_EINVAL;
    SimulationParameters p(4, 4, {shape[0], shape[1], shape[2], shape[3]}, beta, {0, 0, 0, 0}, "torus");
    HBParameters h(config_start, config_stop, therm_steps, or_per_hb, config_sep, data_folder);
    return heatbath_impl(p, h, seed);
}

int lgf_dropin_measure_qdensity(const int shape[4], double beta, int config_start, int config_stop, int flow_steps,
                                double epsilon, int measure_every, const char* data_folder) {
    if (!shape || !data_folder) return LGF_EINVAL;
    SimulationParameters p(4, 4, {shape[0], shape[1], shape[2], shape[3]}, beta, {0, 0, 0, 0}, "torus");
    FlowParameters f(config_start, config_stop, flow_steps, epsilon, measure_every, data_folder);
    return qdensity_impl(p, f);
}

}  // extern "C"
