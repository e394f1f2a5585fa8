// st_tomography_main.cpp -- the ST-Tomography command line of
// gmzang/SpaceTimeTomography (SpaceTimeTomography/main.cpp:13-160), headless:
// the same options, defaults and required arguments, then VolumeData +
// ST_Tomography + Render on the GPU instead of a GLUT window.
//
// Option syntax follows argtable2 as the reference uses it: "-s 0.2",
// "-s0.2", "--Sigma=0.2", "--Sigma 0.2"; options taking several values are
// repeated ("-f 256 -f 256 -f 128").  Options after the reference's set are
// marked "(not in the reference)".
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "ST_Tomography.h"
#include "VolumeData.h"
#include "stt_host.h"

namespace {

struct Opt {
    const char *shortname;  // "" when none
    const char *longname;   // "" when none
    const char *datatype;
    const char *glossary;
    char kind;              // 'd' double, 'i' int, 'f' file, 's' string, 'l' literal
    int mincount, maxcount;
    std::vector<std::string> values;
    int count = 0;
};

std::vector<Opt> make_table() {
    return {
        {"s", "Sigma", "<double>", "Sigma in volume density reconstruction (default as 0.2)", 'd', 0, 1, {}},
        {"t", "Tau", "<double>", "Lambda in volume density reconstruction (default as 0.2)", 'd', 0, 1, {}},
        {"l", "Lambda", "<double>", "TV prior weight in volume density reconstruction ", 'd', 0, 1, {}},
        {"k", "TemporalPrior", "<double>", "temporal prior weight in volume density reconstruction  ", 'd', 0, 1, {}},
        {"e", "Bright constancy prior", "<double>", "Bright constancy weight in volume density reconstruction ", 'd',
         0, 1, {}},
        {"", "huber", "<double>", "trade-off weight for huber norm epsilon ", 'd', 0, 1, {}},
        {"a", "Alpha", "<double>", "stepsize for SART algorithm  (default as 0.3) ", 'd', 0, 1, {}},
        {"o", "", "<output>", "output 3d image (default as \"hello.tif\")", 'f', 0, 1, {}},
        {"i", "projsvolume", "<file>", "Input Dataset file(.mha.tif.tiff 2d bmp and other raw file are supported)",
         'f', 1, 20, {}},
        {"f", "XYZ", "<int>", "takes an integer value (defaults to 9)", 'i', 1, 3, {}},
        {"u", "imgUV", "<int>", "w and h of projection image default:512 ", 'i', 1, 2, {}},
        {"c", "voxelspacing", "<double>", "voxel spacing (default as 1)", 'd', 0, 1, {}},
        {"d", "detector spacing", "<double>", "detector spacing (default as 1)", 'd', 0, 1, {}},
        {"g", "sid", "<double>", " Source to Iso-Object Distance  (default as 600mm)", 'd', 0, 1, {}},
        {"j", "sdd", "<double>", " Source to Detector Distance (default as 1000mm)", 'd', 0, 1, {}},
        {"", "oxyz", "<double>", " offset x y z of the center of volume (default as 0)", 'd', 0, 3, {}},
        {"", "sdg", "<double>", " start degree for each proj sequence", 'd', 0, 20, {}},
        {"v", "nframes", "<int>", "Number of frames", 'i', 0, 1, {}},
        {"r", "nrounds", "<int>", "Number of rounds for each frames", 'i', 0, 1, {}},
        {"b", "AlgorithmIter", "<int>", "Number of algorithm iterations, default as 20", 'i', 0, 1, {}},
        {"p", "SartIter", "<int>", "Number of SART nested iterations, default as 1", 'i', 0, 1, {}},
        {"", "prior", "{STV,SAD,ATV}", "specify the prior you are applying from {STV,SAD,TV} , default as TV", 's', 0,
         1, {}},
        {"", "bp", "{Voxelbased,Raybased}",
         "specify the backprojection methods you are applying from {Voxelbased,Raybased}, default as voxelbased",
         's', 0, 1, {}},
        {"h", "help", "", "print this help and exit", 'l', 0, 1, {}},
        {"", "version", "", "print version information and exit", 'l', 0, 1, {}},
        {"", "joint-iters", "<int>", "joint flow + reconstruction iterations (20) (not in the reference)", 'i', 0, 1,
         {}},
        {"", "pd-passes", "<int>", "primal-dual passes per joint iteration (2) (not in the reference)", 'i', 0, 1, {}},
        {"", "flow-iters", "<int>", "optical-flow iterations per warp (3000) (not in the reference)", 'i', 0, 1, {}},
        {"", "save", "{all,last,none}", "which SART outputs to write (all) (not in the reference)", 's', 0, 1, {}},
        {"", "seed", "<int>", "seed of the SART view order (not in the reference)", 'i', 0, 1, {}},
        {"", "lds", "<file>", "start-angle file (lds.txt) (not in the reference)", 'f', 0, 1, {}},
        {"", "input-dir", "<dir>", "directory of the initial volumes (Input) (not in the reference)", 'f', 0, 1, {}},
        {"", "flow-dir", "<dir>", "directory of the flow outputs (FlowOutput) (not in the reference)", 'f', 0, 1, {}},
        {"", "zero-init", "", "start from zero volumes instead of reading them (not in the reference)", 'l', 0, 1,
         {}},
        {"", "device", "<int>", "CUDA device (0) (not in the reference)", 'i', 0, 1, {}},
    };
}

Opt *find_short(std::vector<Opt> &t, char c) {
    for (Opt &o : t)
        if (o.shortname[0] == c && o.shortname[1] == 0) return &o;
    return nullptr;
}

Opt *find_long(std::vector<Opt> &t, const std::string &name) {
    for (Opt &o : t)
        if (name == o.longname) return &o;
    return nullptr;
}

bool valid_value(const Opt &o, const std::string &v) {
    char *end = nullptr;
    if (o.kind == 'd') {
        std::strtod(v.c_str(), &end);
        return end && *end == 0 && !v.empty();
    }
    if (o.kind == 'i') {
        std::strtol(v.c_str(), &end, 0);
        return end && *end == 0 && !v.empty();
    }
    return true;
}

std::string label(const Opt &o) {
    std::string s;
    if (o.shortname[0]) s += std::string("-") + o.shortname;
    if (o.longname[0]) s += std::string(s.empty() ? "" : "|") + "--" + o.longname;
    return s;
}

void print_syntax(const std::vector<Opt> &t) {
    for (const Opt &o : t) {
        std::string s = label(o);
        if (o.datatype[0]) s += std::string(o.shortname[0] && !o.longname[0] ? " " : "=") + o.datatype;
        if (o.mincount == 0) s = "[" + s + "]";
        if (o.maxcount > 1) s += "...";
        std::printf(" %s", s.c_str());
    }
    std::printf("\n");
}

void print_glossary(const std::vector<Opt> &t) {
    for (const Opt &o : t) {
        std::string s = label(o);
        if (o.datatype[0]) s += " " + std::string(o.datatype);
        std::printf("  %-25s %s\n", s.c_str(), o.glossary);
    }
}

double dval(const Opt &o, double def, int k = 0) { return (int)o.values.size() > k ? std::atof(o.values[k].c_str()) : def; }
int ival(const Opt &o, int def, int k = 0) {
    return (int)o.values.size() > k ? (int)std::strtol(o.values[k].c_str(), nullptr, 0) : def;
}

}  // namespace

int main(int argc, char **argv) {
    const char *progname = "ST-Tomography";
    std::vector<Opt> t = make_table();
    std::vector<std::string> errors;
    for (int a = 1; a < argc; ++a) {
        std::string arg = argv[a];
        Opt *o = nullptr;
        std::string value;
        bool have_value = false;
        if (arg.rfind("--", 0) == 0) {
            std::string name = arg.substr(2);
            const size_t eq = name.find('=');
            if (eq != std::string::npos) {
                value = name.substr(eq + 1);
                name = name.substr(0, eq);
                have_value = true;
            }
            o = find_long(t, name);
            if (!o) {
                errors.push_back("invalid option \"" + arg + "\"");
                continue;
            }
        } else if (arg.size() >= 2 && arg[0] == '-') {
            o = find_short(t, arg[1]);
            if (!o) {
                errors.push_back("invalid option \"" + arg + "\"");
                continue;
            }
            if (arg.size() > 2) {
                value = arg.substr(2);
                have_value = true;
            }
        } else {
            errors.push_back("unexpected argument \"" + arg + "\"");
            continue;
        }
        if (o->kind == 'l') {
            if (have_value) errors.push_back("option " + label(*o) + " takes no value");
            o->count++;
            continue;
        }
        if (!have_value) {
            if (a + 1 >= argc) {
                errors.push_back("option " + label(*o) + " requires an argument");
                continue;
            }
            value = argv[++a];
        }
        if (!valid_value(*o, value)) {
            errors.push_back("invalid argument \"" + value + "\" to option " + label(*o));
            continue;
        }
        if (o->count >= o->maxcount) {
            errors.push_back("excess option " + label(*o));
            continue;
        }
        o->values.push_back(value);
        o->count++;
    }
    Opt &help = *find_long(t, "help"), &version = *find_long(t, "version");
    if (help.count > 0) {
        std::printf("Usage: %s", progname);
        print_syntax(t);
        std::printf("Headless space-time tomography: optical flow and primal-dual reconstruction on the GPU.\n");
        print_glossary(t);
        return 0;
    }
    if (version.count > 0) {
        std::printf("'%s' (libstt %s, sm_100a)\n", progname, stt_version());
        return 0;
    }
    for (const Opt &o : t)
        if (o.count < o.mincount) errors.push_back("missing option " + label(o));
    if (!errors.empty()) {
        for (const std::string &e : errors) std::printf("%s: %s\n", progname, e.c_str());
        std::printf("Try '%s --help' for more information.\n", progname);
        return 1;
    }
    if (argc == 1) {
        std::printf("Try '%s --help' for more information.\n", progname);
        return 0;
    }

    // defaults of main.cpp:64-97
    auto O = [&](const char *name) -> Opt & {
        Opt *o = find_long(t, name);
        if (!o) o = find_short(t, name[0]);
        return *o;
    };
    const double sigma = dval(O("Sigma"), 0.3), tau = dval(O("Tau"), 0.3), lambda = dval(O("Lambda"), 0.1);
    const double tp = dval(O("TemporalPrior"), 0.0), bc = dval(O("Bright constancy prior"), 0.0);
    const double huber = dval(O("huber"), 0.1), alpha = dval(O("Alpha"), 0.1);
    const std::string outfile = find_short(t, 'o')->values.empty() ? "Test/test" : find_short(t, 'o')->values[0];
    const int algo_iter = ival(O("AlgorithmIter"), 2), sart_iter = ival(O("SartIter"), 2);
    const double vs = dval(O("voxelspacing"), 1.0), ds = dval(O("detector spacing"), 1.0);
    const double sdd = dval(O("sdd"), 200.0), sid = dval(O("sid"), 400.0);
    int vols[3] = {ival(O("XYZ"), 63, 0), ival(O("XYZ"), 63, 1), ival(O("XYZ"), 63, 2)};
    int imgwh[2] = {ival(O("imgUV"), 512, 0), 0};
    imgwh[1] = ival(O("imgUV"), imgwh[0], 1);  // one value: a square detector
    double oxyz[3] = {dval(O("oxyz"), 0.0, 0), dval(O("oxyz"), 0.0, 1), dval(O("oxyz"), 0.0, 2)};
    std::vector<double> sdg(20, 0.0);
    for (int k = 0; k < (int)O("sdg").values.size(); ++k) sdg[k] = dval(O("sdg"), 0.0, k);
    const int nframes = ival(O("nframes"), 1), nrounds = ival(O("nrounds"), 1);
    const std::string prior = O("prior").values.empty() ? "ATV" : O("prior").values[0];
    const std::string bp = O("bp").values.empty() ? "Voxelbased" : O("bp").values[0];
    std::vector<const char *> projfiles;
    for (const std::string &f : O("projsvolume").values) projfiles.push_back(f.c_str());
    if (nframes < 1 || nrounds < 1 || vols[0] < 4 || vols[1] < 4 || vols[2] < 4 || imgwh[0] < 2 || imgwh[1] < 2) {
        std::printf("%s: frames, rounds, volume (>= 4) and detector (>= 2) sizes must be positive\n", progname);
        return 1;
    }
    try {
        const int device = ival(O("device"), 0);
        if (stt_host_set_device(device) != 0) throw std::runtime_error(stt_host_last_error());
        VolumeData *data = new VolumeData;
        data->setParas(vols, vs, nframes);
        if (!O("input-dir").values.empty()) data->m_InputDir = O("input-dir").values[0];
        if (O("zero-init").count) {
            int dims[3] = {vols[0], vols[1], vols[2]};
            float sp[3] = {(float)vs, (float)vs, (float)vs};
            data->SetDimensions(dims);
            data->SetSpacings(sp);
            data->_allocate();
        } else {
            data->ReadStructuredFile();
        }
        const int proNo = 10 * nrounds;  // 10 projections per round (main.cpp:147-148)
        ST_Tomography scene(sigma, tau, lambda, tp, bc, huber, outfile.c_str(), imgwh, proNo, algo_iter, sart_iter,
                            alpha, sid, projfiles.data(), oxyz, sdd, ds, prior.c_str(), bp.c_str(), vols, nframes,
                            sdg.data(), nrounds);
        scene.SetDevice(device);
        if (!O("lds").values.empty()) scene.SetLdsFile(O("lds").values[0]);
        scene.SetJointIterations(ival(O("joint-iters"), 20));
        scene.SetPrimalDualPasses(ival(O("pd-passes"), 2));
        scene.SetFlowIterations(ival(O("flow-iters"), 3000));
        if (!O("seed").values.empty()) scene.SetSeed((unsigned long long)ival(O("seed"), 0));
        if (!O("flow-dir").values.empty()) scene.SetFlowDirectory(O("flow-dir").values[0]);
        const std::string save = O("save").values.empty() ? "all" : O("save").values[0];
        scene.SetSaveMode(save == "last" ? ST_Tomography::SAVE_LAST
                                         : (save == "none" ? ST_Tomography::SAVE_NONE : ST_Tomography::SAVE_ALL));
        scene.SetData(data);
        scene.Render();
        delete data;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "%s: %s\n", progname, e.what());
        return 2;
    }
    return 0;
}
