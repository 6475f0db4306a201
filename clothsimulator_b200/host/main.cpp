// clothsim: command line of the --gpu path, with the reference's argument order (main.cu:9-33):
//   clothsim simulate_offline <config.json> <output dir> --gpu
//   clothsim resume_offline <output dir> --gpu
// The interactive modes (simulate, resume, replay) need OpenGL and are unavailable here.  The
// reference's CPU path (no --gpu) is the reference itself; this program only provides --gpu.
#include <cstring>
#include <iostream>

extern "C" int cs_sim_run(const char* mode, const char* path, const char* dir, int device, int* steps);
extern "C" const char* cs_sim_last_error();

int main(int argc, char** argv) {
    if (argc < 3) {
        std::cerr << "Please enter mode and configuration file path" << std::endl;
        return 1;
    }
    const std::string mode = argv[1];
    bool gpu = false;
    for (int i = 2; i < argc; i++)
        if (std::strcmp(argv[i], "--gpu") == 0) gpu = true;
    if (!gpu) {
        std::cerr << "this build provides the --gpu path only; run the reference for its CPU path" << std::endl;
        return 1;
    }
    int st;
    if (mode == "simulate_offline") {
        if (argc < 5) {
            std::cerr << "usage: clothsim simulate_offline <config.json> <output dir> --gpu" << std::endl;
            return 1;
        }
        st = cs_sim_run("simulate_offline", argv[2], argv[3], 0, nullptr);
    } else if (mode == "resume_offline") {
        st = cs_sim_run("resume_offline", "", argv[2], 0, nullptr);
    } else {
        st = cs_sim_run(mode.c_str(), argv[2], "", 0, nullptr);
    }
    if (st != 0) {
        std::cerr << cs_sim_last_error() << std::endl;
        return 1;
    }
    return 0;
}
