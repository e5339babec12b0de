// deck.cpp — the muMatScale input-deck format, parsed into mms_params.
//
// Follows set_defaults (read_ctrl.c:29-108) and read_config
// (read_ctrl.c:234-812): whitespace keyword lines read in 255-character
// chunks, keywords case-insensitive, '#' / '%' comment lines, arguments
// scanned with the same sscanf conversions (so trailing "/* ... */" text is
// ignored the same way), unknown keywords ignored, include files for
// GeoFileName / MatFileName / AlloyPropsFile0.  Where the reference aborts
// (a failed assert on an argument count, CalculationModel, an unknown
// TemperatureModel or DataFormat) this returns MMS_ERR_DECK.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <strings.h>
#include <vector>

#include "mms_internal.h"

namespace {

struct Lists {
    std::vector<mms_fixed_nuc> fixed;
    std::vector<mms_nuc_volume> volumes;
};

mms_status parse_file(const char *path, mms_params *bp, Lists &lists, int depth, std::string &err)
{
    if (depth > 16) {
        err = "include depth exceeded";
        return MMS_ERR_DECK;
    }
    FILE *fp = std::fopen(path, "r");
    if (!fp) {
        err = std::string("Unable to open control file: ") + path;
        return MMS_ERR_DECK;
    }
    const int MAX_STRING_LEN = 256;  // globals.h:53
    char line[MAX_STRING_LEN + 2];
    char token[MAX_STRING_LEN + 2];
    char strarg[MAX_STRING_LEN + 2];
    mms_status st = MMS_OK;
    auto need = [&](int c, int n, const char *kw) {
        if (c != n) {
            err = std::string("bad arguments for ") + kw;
            st = MMS_ERR_DECK;
            return false;
        }
        return true;
    };
    while (st == MMS_OK && std::fgets(line, MAX_STRING_LEN, fp) != nullptr) {
        int idx = 0;
        char *lp = line;
        int c = std::sscanf(lp, " %s%n", token, &idx);
        if (c <= 0 || token[0] == '#' || token[0] == '%') continue;
        lp += idx;
        auto is = [&](const char *kw) { return strcasecmp(token, kw) == 0; };
        if (is("BaseFileName")) {
            c = std::sscanf(lp, "%255s", bp->basefilename);
            need(c, 1, token);
        } else if (is("NSubblocks")) {
            need(std::sscanf(lp, "%d %d %d", &bp->gnsbx, &bp->gnsby, &bp->gnsbz), 3, token);
        } else if (is("NCellsPerSB")) {
            need(std::sscanf(lp, "%d %d %d", &bp->gsdimx, &bp->gsdimy, &bp->gsdimz), 3, token);
        } else if (is("CellSize")) {
            need(std::sscanf(lp, "%lf", &bp->cellSize), 1, token);
        } else if (is("CourantLimit")) {
            need(std::sscanf(lp, "%lf", &bp->courant_limit), 1, token);
        } else if (is("FaceCtrl")) {
            int x, y, z;
            c = std::sscanf(lp, "%d %d %d %d %d %d", &bp->padBndyX, &x, &bp->padBndyY, &y,
                            &bp->padBndyZ, &z);
            if (need(c, 6, token) && (bp->padBndyX != x || bp->padBndyY != y || bp->padBndyZ != z)) {
                err = "FaceCtrl: both faces of an axis must match";
                st = MMS_ERR_DECK;
            }
        } else if (is("FixedNuc")) {
            mms_fixed_nuc f;
            c = std::sscanf(lp, "%lf %lf %lf %lf %lf %lf %lf", &f.x, &f.y, &f.z, &f.ax, &f.ay,
                            &f.az, &f.threshold);
            if (need(c, 7, token)) lists.fixed.push_back(f);
        } else if (is("NucVolume")) {
            mms_nuc_volume v;
            c = std::sscanf(lp, "%lg %lg %lg %lg %lg %lg %lg %lg\n", &v.density, &v.minx, &v.miny,
                            &v.minz, &v.maxx, &v.maxy, &v.maxz, &v.threshold);
            if (need(c, 8, token)) {
                v.density = v.density / 100.0;
                lists.volumes.push_back(v);
            }
        } else if (is("MaxGrainDensity")) {
            need(std::sscanf(lp, "%lf", &bp->maxGrainDensity), 1, token);
        } else if (is("MaxGrainDensitySurf")) {
            need(std::sscanf(lp, "%lf", &bp->maxGrainDensitySurf), 1, token);
        } else if (is("MaxTotGrains")) {
            unsigned long v = 0;
            if (need(std::sscanf(lp, "%lu", &v), 1, token)) bp->maxTotalGrains = v;
        } else if (is("RandomizeGrains")) {
            need(std::sscanf(lp, "%d", &bp->randomize_grains), 1, token);
        } else if (is("MouldNuc") || is("MoldNuc")) {
            need(std::sscanf(lp, "%d", &bp->doSurfaceNuc), 1, token);
        } else if (is("GNGaussCentre") || is("GNGaussCenter")) {
            need(std::sscanf(lp, "%lf", &bp->gnGaussCenter), 1, token);
        } else if (is("GNGaussSigma")) {
            need(std::sscanf(lp, "%lf", &bp->gnGaussSigma), 1, token);
        } else if (is("GNGaussCentreSurf") || is("GNGaussCenterSurf")) {
            need(std::sscanf(lp, "%lf", &bp->gnGaussCenterSurf), 1, token);
        } else if (is("GNGaussSigmaSurf")) {
            need(std::sscanf(lp, "%lf", &bp->gnGaussSigmaSurf), 1, token);
        } else if (is("GNOriented")) {
            need(std::sscanf(lp, "%d", &bp->gnUseOrientation), 1, token);
        } else if (is("LiquidusTemp")) {
            need(std::sscanf(lp, "%lf", &bp->liquidusTemp), 1, token);
        } else if (is("SolidusTemp")) {
            need(std::sscanf(lp, "%lf", &bp->solidusTemp), 1, token);
        } else if (is("T_pure")) {
            double v;
            need(std::sscanf(lp, "%lf", &v), 1, token);
        } else if (is("Cinit")) {
            need(std::sscanf(lp, "%lf", &bp->Cinit), 1, token);
        } else if (is("m_solute0")) {
            c = std::sscanf(lp, "%lf %lf %lf", &bp->m_solute0_a, &bp->m_solute0_b, &bp->m_solute0_c);
            bp->m_solute0 = bp->m_solute0_c;
            need(c, 3, token);
        } else if (is("part_coef0")) {
            c = std::sscanf(lp, "%lf %lf %lf", &bp->part_coef_a, &bp->part_coef_b, &bp->part_coef_c);
            bp->part_coef = bp->part_coef_c;
            need(c, 3, token);
        } else if (is("Dsol")) {
            need(std::sscanf(lp, "%lf", &bp->Dsol), 1, token);
        } else if (is("Dliq")) {
            need(std::sscanf(lp, "%lf", &bp->Dliq), 1, token);
        } else if (is("CalculationModel")) {
            err = "Unknown Calculation Model (read_ctrl.c:428-438 always rejects this keyword)";
            st = MMS_ERR_DECK;
        } else if (is("TemperatureModel")) {
            c = std::sscanf(lp, "%255s", strarg);
            if (need(c, 1, token) && strcasecmp(strarg, "INTERNAL") != 0) {
                err = std::string("Unknown Temperature Model '") + strarg + "'";
                st = MMS_ERR_DECK;
            }
        } else if (is("ExternalTempFile") || is("ProcastMaterialGroup") ||
                   is("CalculateProcastRegion") || is("ProcastRegion") || is("GradSlope") ||
                   is("Slope_coef") || is("Iso_Coef_One") || is("Iso_coef_Two") ||
                   is("Coef_Iso2") || is("GG_Constant") || is("GG_Cub") ||
                   is("ProfileWriteFreq") || is("FluidFlowMode") || is("FluidFlowTimeStep") ||
                   is("FFStartTime") || is("FFStepGap") || is("Viscosity") ||
                   is("ThermExpCoe") || is("SoluteExpCoe") || is("ReferenceTemp") ||
                   is("ReferSolute") || is("Gravity_x") || is("Gravity_y") || is("Gravity_z") ||
                   is("InitialVelocity") || is("SemiaxisSide") || is("SemiaxisDepth") ||
                   is("SemiaxisRear") || is("SemiaxisFront")) {
            // accepted by the reference but not read on the CA hot path
            double a, b, cc;
            int n = std::sscanf(lp, "%lf %lf %lf", &a, &b, &cc);
            (void)n;
        } else if (is("TipCurvature")) {
            need(std::sscanf(lp, "%d", &bp->tip_curv), 1, token);
        } else if (is("GibbsThomsonCoef")) {
            need(std::sscanf(lp, "%lg", &bp->gibbs_coef), 1, token);
        } else if (is("InitialTemperature")) {
            need(std::sscanf(lp, "%lf", &bp->initialTemperature), 1, token);
        } else if (is("Velo_Coef")) {
            need(std::sscanf(lp, "%lf", &bp->velo_coef), 1, token);
        } else if (is("Grad_Coef")) {
            need(std::sscanf(lp, "%lf", &bp->grad_coef), 1, token);
        } else if (is("Gradient")) {
            need(std::sscanf(lp, "%lf", &bp->gradient), 1, token);
        } else if (is("Velocity")) {
            need(std::sscanf(lp, "%lf", &bp->velocity), 1, token);
        } else if (is("CoolingRate")) {
            need(std::sscanf(lp, "%lf", &bp->cool_rate), 1, token);
        } else if (is("FSGrow")) {
            c = std::sscanf(lp, "%lf", &bp->fsgrow);
            bp->rev_fsgrow = 1.0 / bp->fsgrow;
            need(c, 1, token);
        } else if (is("TimeStep")) {
            need(std::sscanf(lp, "%lf", &bp->ts_delt), 1, token);
        } else if (is("FinishTime")) {
            need(std::sscanf(lp, "%lf", &bp->finish_time), 1, token);
        } else if (is("FsFinish")) {
            need(std::sscanf(lp, "%lf", &bp->fs_finish), 1, token);
        } else if (is("ScreenPFreq")) {
            need(std::sscanf(lp, "%d", &bp->screenpfreq), 1, token);
        } else if (is("DataWriteFreq")) {
            need(std::sscanf(lp, "%d", &bp->data_write_freq), 1, token);
        } else if (is("DataWriteStart")) {
            // read_ctrl.c:594-600 stores the value in both fields: the data
            // write start and the checkpoint frequency (the reference has no
            // keyword of its own for the latter)
            need(std::sscanf(lp, "%d", &bp->data_write_start), 1, token);
            bp->checkpoint_freq = bp->data_write_start;
        } else if (is("DataFormat")) {
            c = std::sscanf(lp, "%255s", strarg);
            if (need(c, 1, token)) {
                if (strcasecmp(strarg, "VTK") == 0) bp->vis_format = 1;
                else if (strcasecmp(strarg, "XDMF") == 0) bp->vis_format = 2;
                else {
                    err = std::string("Unsupported data file type: ") + strarg;
                    st = MMS_ERR_DECK;
                }
            }
        } else if (is("GeoFileName") || is("MatFileName") || is("AlloyPropsFile0")) {
            c = std::sscanf(lp, "%255s", strarg);
            if (need(c, 1, token)) st = parse_file(strarg, bp, lists, depth + 1, err);
        } else if (is("RandSeedVal")) {
            need(std::sscanf(lp, "%u", &bp->base_random_seed), 1, token);
        } else if (is("Density")) {
            need(std::sscanf(lp, "%lf", &bp->rho), 1, token);
        } else if (is("AnalyticalThermal")) {
            if (need(std::sscanf(lp, "%d", &bp->thermal_ana), 1, token) && bp->thermal_ana) bp->am = 1;
        } else if (is("LaserPower")) {
            need(std::sscanf(lp, "%lf", &bp->lpow), 1, token);
        } else if (is("LaserSpeed")) {
            need(std::sscanf(lp, "%lf", &bp->lv), 1, token);
        } else if (is("LaserSpotSize")) {
            need(std::sscanf(lp, "%lf", &bp->lsd), 1, token);
        } else if (is("LaserAbsorption")) {
            need(std::sscanf(lp, "%lf", &bp->lab), 1, token);
        } else if (is("LaserHatchSpacing")) {
            need(std::sscanf(lp, "%lf", &bp->lhs), 1, token);
        } else if (is("SubInitialTemp")) {
            need(std::sscanf(lp, "%lf", &bp->liniT), 1, token);
        } else if (is("ThermalConductivity")) {
            need(std::sscanf(lp, "%lf", &bp->lthcon), 1, token);
        } else if (is("SpecificHeat")) {
            need(std::sscanf(lp, "%lf", &bp->lcp), 1, token);
        } else if (is("LaserStartLocation")) {
            need(std::sscanf(lp, "%lf %lf %lf", &bp->x0, &bp->y0, &bp->z0), 3, token);
        } else if (is("NoOfLayers")) {
            need(std::sscanf(lp, "%d", &bp->amlayer), 1, token);
        } else if (is("NoOfTracks")) {
            need(std::sscanf(lp, "%d", &bp->amtracks), 1, token);
        }
    }
    std::fclose(fp);
    return st;
}

}  // namespace

extern "C" mms_status mms_params_default(mms_params *bp)
{
    if (!bp) return MMS_ERR_ARG;
    std::memset(bp, 0, sizeof(*bp));  // xmalloc zero-fills bp (ca_main.c:91)
    std::snprintf(bp->basefilename, sizeof bp->basefilename, "output");
    bp->padBndyX = bp->padBndyY = bp->padBndyZ = 1;
    bp->cellSize = 0.01f;  // float literals kept as in read_ctrl.c:37-61
    bp->initialTemperature = 100.0f;
    bp->cool_rate = 0.0f;
    bp->liquidusTemp = 1180.0f;
    bp->solidusTemp = 1120.0f;
    bp->courant_limit = 0.2;
    bp->tip_curv = 0;
    bp->gibbs_coef = 0.0;
    bp->base_random_seed = (unsigned int)std::time(nullptr);
    bp->fs_finish = 1.0f;
    bp->finish_time = 0.0f;
    bp->ts_delt = 0.1f;
    bp->screenpfreq = 1;
    bp->vis_format = 0;
    bp->data_write_freq = 0;
    bp->data_write_start = 0;
    bp->randomize_grains = 1;
    bp->maxGrainDensity = 0.0;
    bp->gnGaussCenter = 0.0;
    bp->gnGaussSigma = 0.0;
    bp->gnUseOrientation = 0;
    bp->maxGrainDensitySurf = 0.0;
    bp->gnGaussCenterSurf = 0.0;
    bp->gnGaussSigmaSurf = 0.0;
    bp->maxTotalGrains = (uint64_t)1e6;
    bp->doSurfaceNuc = 1;
    bp->m_solute0 = -2.0;
    bp->m_solute0_a = 0.0;
    bp->m_solute0_b = 0.0;
    bp->m_solute0_c = -2.0;
    bp->Cinit = 5.0;
    bp->Dsol = 1e-13;
    bp->Dliq = 1e-9;
    bp->part_coef = 0.3;
    bp->part_coef_a = 0.0;
    bp->part_coef_b = 0.0;
    bp->part_coef_c = 0.3;
    bp->am = 0;
    bp->thermal_ana = 0;
    bp->amlayer = 1;
    bp->amtracks = 1;
    bp->precision = MMS_PREC_F64;
    bp->device = 0;
    return MMS_OK;
}

extern "C" mms_status mms_deck_read(const char *path, mms_params *bp)
{
    if (!path || !bp) return MMS_ERR_ARG;
    Lists lists;
    for (int i = 0; i < bp->n_fixed_nucs; i++) lists.fixed.push_back(bp->fixed_nucs[i]);
    for (int i = 0; i < bp->n_nuc_volumes; i++) lists.volumes.push_back(bp->nuc_volumes[i]);
    std::string err;
    mms_status st = parse_file(path, bp, lists, 0, err);
    if (st != MMS_OK) {
        std::fprintf(stderr, "mms_deck_read: %s\n", err.c_str());
        return st;
    }
    mms_params_free_lists(bp);
    if (!lists.fixed.empty()) {
        auto *f = (mms_fixed_nuc *)std::malloc(sizeof(mms_fixed_nuc) * lists.fixed.size());
        std::memcpy(f, lists.fixed.data(), sizeof(mms_fixed_nuc) * lists.fixed.size());
        bp->fixed_nucs = f;
        bp->n_fixed_nucs = (int)lists.fixed.size();
    }
    if (!lists.volumes.empty()) {
        auto *v = (mms_nuc_volume *)std::malloc(sizeof(mms_nuc_volume) * lists.volumes.size());
        std::memcpy(v, lists.volumes.data(), sizeof(mms_nuc_volume) * lists.volumes.size());
        bp->nuc_volumes = v;
        bp->n_nuc_volumes = (int)lists.volumes.size();
    }
    return MMS_OK;
}

extern "C" void mms_params_free_lists(mms_params *bp)
{
    if (!bp) return;
    std::free((void *)bp->fixed_nucs);
    std::free((void *)bp->nuc_volumes);
    bp->fixed_nucs = nullptr;
    bp->nuc_volumes = nullptr;
    bp->n_fixed_nucs = 0;
    bp->n_nuc_volumes = 0;
}

extern "C" size_t mms_params_size(void) { return sizeof(mms_params); }
