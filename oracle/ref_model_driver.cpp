// Test-only driver of the reference solver, compiled with the reference's own
// sources by oracle/Makefile (output in oracle/_ref/).  It runs
// Algorithm::solve in-process with a dosage model set in Settings: the
// reference's command line cannot reach that path (src/main.cpp:161 rejects
// the argument-less -j/-k/-l, and -z/-y never store their file name,
// src/main.cpp:341-358), while its reader implements the models
// (src/AIOwrapper.cpp:257-340, 1213-1275).
//
//   ref_model_driver XL XR Y OUT NGPRED MODEL [FACTORS|-] [-b] [-f] [-i] [-v INTER | -w INTER] [-t THREADS]
//                    [-k] [-x EXCLUDE]
//
// MODEL is the reference's Settings::model: 0 additive, 1 dominant,
// 2 recessive, 3 custom linear, 4 custom additive, -1 none.  -v sets the
// single-set interactions with the file INTER (keeping the SNP column, as
// the reference's -v does, src/main.cpp:369-378), -w one analysis per
// interaction column (src/main.cpp:380-389); the command-line forms of both
// store atof(optarg) as the file name (src/main.cpp:370, 381).
#include <cstdlib>
#include <cstring>
#include <iostream>

#include "Algorithm.h"

int main(int argc, char** argv) {
    if (argc < 7) {
        std::cout << "usage: ref_model_driver XL XR Y OUT NGPRED MODEL [FACTORS|-] [-b] [-f] [-i]" << std::endl;
        return 2;
    }
    Settings params;
    Algorithm alg;
    alg.applyDefaultParams(params);
    params.fnameAL = argv[1];
    params.fnameAR = argv[2];
    params.fnameY = argv[3];
    params.fnameOutFiles = argv[4];
    params.r = std::atoi(argv[5]);
    params.model = std::atoi(argv[6]);
    params.dosages = params.model >= 0;
    int a = 7;
    bool keep_dep = true;   // -k: interactions without the SNP column itself (the reference's keep_depVar = false)
    if (a < argc && argv[a][0] != '-') params.fname_dosages = argv[a++];
    else if (a < argc && std::strcmp(argv[a], "-") == 0) ++a;
    for (; a < argc; ++a) {
        if (!std::strcmp(argv[a], "-b")) params.storeBin = true;
        else if (!std::strcmp(argv[a], "-f")) params.storePInd = true;
        else if (!std::strcmp(argv[a], "-i")) params.disp_cov = true;
        else if (!std::strcmp(argv[a], "-t") && a + 1 < argc) params.threads = std::atoi(argv[++a]);
        else if (!std::strcmp(argv[a], "-x") && a + 1 < argc) params.fname_excludelist = argv[++a];
        else if (!std::strcmp(argv[a], "-k")) keep_dep = false;
        else if (!std::strcmp(argv[a], "-v") && a + 1 < argc) {
            params.fname_interactions = argv[++a];
            params.use_interactions = true;
            params.keep_depVar = true;
            params.use_multiple_interaction_sets = false;
        } else if (!std::strcmp(argv[a], "-w") && a + 1 < argc) {
            params.fname_interactions = argv[++a];
            params.use_interactions = true;
            params.keep_depVar = true;
            params.use_multiple_interaction_sets = true;
        }
    }
    if (params.use_interactions) params.keep_depVar = keep_dep;
    blas_set_num_threads(params.threads);
    Outputs out = {0};
    alg.solve(params, out, P_NEQ_B_OPT_MD);
    std::cout << std::endl << "Number of Significant Results: " << out.total_sig_results << std::endl;
    return 0;
}
