/*
 * lgf_dropin.h — drop-in replacement for the LGF reference's flow workflows.
 *
 * C++ callers keep the reference's parameter classes and entry points:
 *   SimulationParameters(NrDims, extdofs, shape, beta, cuts, LatticeType)
 *       (LGF/SimulationParameters.h:3-47)
 *   FlowParameters(start, stop, flowSteps, epsilon, measureEvery, dataFolder)
 *       (LGF/SimulationParameters.h:49-86)
 *   void FlowSavedGaugeConfigurations(SimulationParameters&, FlowParameters&)
 *       (LGF/LGF.h:31, LGF/LGF.cpp:163-196)
 *   void ResumeFlowedConfiguration(SimulationParameters&, FlowParameters&, double)
 *       (LGF/LGF.h:32, LGF/LGF.cpp:197-226)
 *   void MeasureQdensityDistribution(SimulationParameters&, FlowParameters&)
 *       (LGF/LGF.h:35, LGF/LGF.cpp:114-124)
 *   void MeasureFlowedGaugeConfigurations(SimulationParameters&, FlowParameters&)
 *       (LGF/LGF.h:34, LGF/LGF.cpp:228-255)
 *   HBParameters(start, stop, ThermSteps, OR_per_HB, configSep, dataFolder)
 *       (LGF/SimulationParameters.h:88-124) and
 *   void GenerateHeatBathGaugeConfigurations(SimulationParameters&, HBParameters&)
 *       (LGF/LGF.h:29, LGF/LGF.cpp:136-160), the input generator
 * with the same input/output files (ensembles/.../*.bin, Observables/.../*.csv)
 * and the same stdout lines; the flow and the measurements run on the GPU
 * through lgf_b200.h.  Other languages bind the extern "C" functions at the end.
 *
 * Engine selection (no reference counterpart): LGF_PRECISION=fp64|fp32mixed
 * (default fp64, the plain form) and LGF_DEVICE=<cuda device> in the
 * environment, or lgf_dropin_configure().
 */
#ifndef LGF_DROPIN_H
#define LGF_DROPIN_H

#include <stdint.h>

#ifdef __cplusplus
#include <string>
#include <vector>

class SimulationParameters {
public:
    /* LatticeType must be "torus" or "torus_OpenT" (LGF/SimulationParameters.h:12-19);
     * anything else prints the reference's message and exits with EXIT_FAILURE.
     * The engine flows "torus" only; "torus_OpenT" is rejected at flow time. */
    SimulationParameters(int NrDims, int extdofs, std::vector<int> shape, double beta, std::vector<int> cuts,
                         std::string LatticeType = "torus");
    int getNrDims() { return m_NrDims; }
    int getextdofs() { return m_extdofs; }
    int getshape(int i) { return m_shape[i]; }
    double getbeta() { return m_beta; }
    int getcuts(int i) { return m_cuts[i]; }
    std::string getLatticeType() { return m_LatticeType; }

private:
    int m_NrDims;
    int m_extdofs;
    std::vector<int> m_shape;
    double m_beta;
    std::vector<int> m_cuts;
    std::string m_LatticeType;
};

class FlowParameters {
public:
    FlowParameters(int ConfigurationStart, int ConfigurationStop, int flowSteps, double epsilon,
                   int measure_every_nth_step, const std::string& dataFolder)
        : m_ConfigurationStart(ConfigurationStart), m_ConfigurationStop(ConfigurationStop), m_flowSteps(flowSteps),
          m_epsilon(epsilon), m_measure_every_nth_step(measure_every_nth_step), m_dataFolder(dataFolder) {}
    int getConfigurationStart() { return m_ConfigurationStart; }
    int getConfigurationStop() { return m_ConfigurationStop; }
    int getflowSteps() { return m_flowSteps; }
    double getepsilon() { return m_epsilon; }
    int getMeasuringInterval() { return m_measure_every_nth_step; }
    std::string getdataFolder() { return m_dataFolder; }

private:
    int m_ConfigurationStart;
    int m_ConfigurationStop;
    int m_flowSteps;
    double m_epsilon;
    int m_measure_every_nth_step;
    std::string m_dataFolder;
};

class HBParameters {
public:
    HBParameters(int ConfigurationStart, int ConfigurationStop, int ThermSteps, int OR_per_HB, int configSep,
                 const std::string& dataFolder)
        : m_ConfigurationStart(ConfigurationStart), m_ConfigurationStop(ConfigurationStop), m_ThermSteps(ThermSteps),
          m_OR_per_HB(OR_per_HB), m_configSep(configSep), m_dataFolder(dataFolder) {}
    int getConfigurationStart() { return m_ConfigurationStart; }
    int getConfigurationStop() { return m_ConfigurationStop; }
    int getThermSteps() { return m_ThermSteps; }
    int getOR_per_HB() { return m_OR_per_HB; }
    int getconfigSep() { return m_configSep; }
    std::string getdataFolder() { return m_dataFolder; }

private:
    int m_ConfigurationStart;
    int m_ConfigurationStop;
    int m_ThermSteps;
    int m_OR_per_HB;
    int m_configSep;
    std::string m_dataFolder;
};

void FlowSavedGaugeConfigurations(SimulationParameters& params, FlowParameters& flowParams);
/* GenerateHeatBathGaugeConfigurations (LGF/LGF.cpp:136-160) on the GPU; the
 * generator seed comes from LGF_SEED in the environment, else std::random_device
 * (the reference's default, LGF/Math/Random.h:18-22). */
void GenerateHeatBathGaugeConfigurations(SimulationParameters& params, HBParameters& HBparams);
void ResumeFlowedConfiguration(SimulationParameters& params, FlowParameters& flowParams, double flowTime_pickup);
void MeasureQdensityDistribution(SimulationParameters& params, FlowParameters& flowParams);
void MeasureFlowedGaugeConfigurations(SimulationParameters& params, FlowParameters& flowParams);

extern "C" {
#endif

/* precision: LGF_PREC_FP64 (0) or LGF_PREC_FP32MIXED (1); reunit_every applies
 * to the mixed form (0 = never); device = CUDA device ordinal */
int lgf_dropin_configure(int precision, int reunit_every, int device);
/* FlowSavedGaugeConfigurations flows up to `configs` saved configurations
 * together through lgf_batch_run (1 = one by one, the default; the
 * environment variable LGF_BATCH sets it too) and writes the same stdout
 * lines, CSV rows and flowed files, in the same order, with the same values
 * bit for bit.  No reference counterpart (the reference flows one at a time,
 * LGF/LGF.cpp:169-195). */
int lgf_dropin_set_batch(int configs);

/* Flat C entry points with the reference's arguments (for cgo/ctypes/JNI).
 * Return 0 on success, a negative LGF_E* status when a configuration failed
 * (the remaining configurations are still processed). */
int lgf_dropin_flow_saved(const int shape[4], double beta, int config_start, int config_stop, int flow_steps,
                          double epsilon, int measure_every, const char* data_folder);
int lgf_dropin_resume_flowed(const int shape[4], double beta, int config_start, int config_stop, int flow_steps,
                             double epsilon, int measure_every, const char* data_folder, double flow_time_pickup);
int lgf_dropin_measure_qdensity(const int shape[4], double beta, int config_start, int config_stop, int flow_steps,
                                double epsilon, int measure_every, const char* data_folder);
int lgf_dropin_measure_flowed(const int shape[4], double beta, int config_start, int config_stop, int flow_steps,
                              double epsilon, int measure_every, const char* data_folder);
int lgf_dropin_generate_heatbath(const int shape[4], double beta, int config_start, int config_stop, int therm_steps,
                                 int or_per_hb, int config_sep, const char* data_folder, uint64_t seed);

#ifdef __cplusplus
}
#endif
#endif
