// params.cpp -- icy::SimParams host logic behind the C ABI.
//
// Restates simulation/parameters_sim.cpp: Reset (:5-56), ParseFile
// (:59-119), ComputeLame (:121-126), ComputeHelperVariables (:128-136),
// ComputeCamClayParams2 (:138-147), ComputeIntegerBlockCoords (:149-155).
// The reference parses with rapidjson, which is not part of this build; the
// configuration files are flat JSON objects, so a small reader for objects of
// string / number / literal values stands in for it.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <map>

#include "../../include/icempm.h"
#include "errors.h"

extern "C" void icm_params_compute_lame(icy_SimParams *p)
{
    p->lambda = p->YoungsModulus * p->PoissonsRatio / ((1 + p->PoissonsRatio) * (1 - 2 * p->PoissonsRatio));
    p->mu = p->YoungsModulus / (2 * (1 + p->PoissonsRatio));
    p->kappa = p->mu * 2. / 3. + p->lambda;
}

extern "C" void icm_params_compute_helpers(icy_SimParams *p)
{
    p->UpdateEveryNthStep = (int)(1.f / (200 * p->InitialTimeStep));
    p->cellsize = p->GridXDimension / p->GridX;
    p->cellsize_inv = 1. / p->cellsize;
    p->Dp_inv = 4. / (p->cellsize * p->cellsize);
    p->IndRSq = p->IndDiameter * p->IndDiameter / 4.;
    p->GridTotal = p->GridX * p->GridY;
}

extern "C" void icm_params_compute_camclay(icy_SimParams *p)
{
    icm_params_compute_lame(p);
    p->NACC_beta = p->IceTensileStrength / p->IceCompressiveStrength;
    const double beta = p->NACC_beta;
    const double q = p->IceShearStrength;
    const double p0 = p->IceCompressiveStrength;
    p->NACC_M = (2 * q * std::sqrt(1 + 2 * beta)) / (p0 * (1 + beta));
    p->NACC_Msq = p->NACC_M * p->NACC_M;
}

extern "C" void icm_params_compute_block_coords(icy_SimParams *p)
{
    p->nxmin = (int)std::floor(p->xmin / p->cellsize);
    p->nxmax = (int)std::ceil(p->xmax / p->cellsize);
    p->nymin = (int)std::floor(p->ymin / p->cellsize);
    p->nymax = (int)std::ceil(p->ymax / p->cellsize);
}

extern "C" void icm_params_reset(icy_SimParams *p)
{
    std::memset(p, 0, sizeof(*p));
    p->grid_array = nullptr;
    p->pts_array = nullptr;
    p->indenter_force_accumulator = nullptr;
    p->nPts = 0;
    p->n_indenter_subdivisions = 100;
    p->InitialTimeStep = 3.e-5;
    p->YoungsModulus = 5.e8;
    p->GridX = 128;
    p->GridY = 55;
    p->ParticleViewSize = 2.5f;
    p->GridXDimension = 3.33;
    p->SimulationEndTime = 12;
    p->PoissonsRatio = 0.3;
    p->Gravity = 9.81;
    p->Density = 980;
    p->IndDiameter = 0.324;
    p->IndVelocity = 0.2;
    p->IndDepth = 0.25;
    p->SimulationStep = 0;
    p->SimulationTime = 0;
    p->IceCompressiveStrength = 100e6;
    p->IceTensileStrength = 1e6;
    p->IceShearStrength = 0.5e6;
    p->DP_tan_phi = std::tan(30 * ICM_PI / 180.);
    p->DP_threshold_p = 1e3;
    p->tpb_P2G = 256;
    p->tpb_Upd = 512;
    p->tpb_G2P = 128;
    p->indenter_x = p->indenter_x_initial = p->indenter_y = p->indenter_y_initial = 0;
    p->SetupType = 0;
    p->GrainVariability = 0.50;
    p->UseWarpLevelReduction = 0;
    p->SortPointsByGridCell = 1;
    icm_params_compute_lame(p);
    icm_params_compute_camclay(p);
    icm_params_compute_helpers(p);
}

extern "C" size_t icm_pitch_elems(size_t n) { return (n + 63) / 64 * 64; }

// ------------------------------------------------------- flat JSON reader

namespace {

struct JVal {
    enum Kind { NUM, STR, LIT } kind;
    double num;
    bool is_int;
    std::string str;
};

struct Reader {
    const char *s;
    size_t i, n;
    std::string err;
    void ws()
    {
        while (i < n && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) i++;
    }
    bool str(std::string &out)
    {
        if (i >= n || s[i] != '"') return false;
        i++;
        out.clear();
        while (i < n && s[i] != '"') {
            char c = s[i++];
            if (c == '\\') {
                if (i >= n) return false;
                char e = s[i++];
                switch (e) {
                case 'n': out += '\n'; break;
                case 't': out += '\t'; break;
                case 'r': out += '\r'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'u':
                    if (i + 4 > n) return false;
                    out += '?';
                    i += 4;
                    break;
                default: out += e; break;
                }
            } else {
                out += c;
            }
        }
        if (i >= n) return false;
        i++;
        return true;
    }
    bool value(JVal &v)
    {
        ws();
        if (i >= n) return false;
        if (s[i] == '"') {
            v.kind = JVal::STR;
            return str(v.str);
        }
        if (s[i] == '{' || s[i] == '[') {
            err = "nested values are not supported";
            return false;
        }
        if (!std::strncmp(s + i, "true", 4) || !std::strncmp(s + i, "null", 4)) {
            v.kind = JVal::LIT;
            v.num = s[i] == 't' ? 1 : 0;
            v.is_int = true;
            i += 4;
            return true;
        }
        if (!std::strncmp(s + i, "false", 5)) {
            v.kind = JVal::LIT;
            v.num = 0;
            v.is_int = true;
            i += 5;
            return true;
        }
        size_t j = i;
        bool frac = false;
        if (j < n && (s[j] == '-' || s[j] == '+')) j++;
        while (j < n && ((s[j] >= '0' && s[j] <= '9') || s[j] == '.' || s[j] == 'e' || s[j] == 'E' || s[j] == '-' ||
                         s[j] == '+')) {
            if (s[j] == '.' || s[j] == 'e' || s[j] == 'E') frac = true;
            j++;
        }
        if (j == i) return false;
        std::string tok(s + i, j - i);
        char *end = nullptr;
        v.num = std::strtod(tok.c_str(), &end);
        if (!end || *end) return false;
        v.kind = JVal::NUM;
        v.is_int = !frac;
        i = j;
        return true;
    }
    bool object(std::map<std::string, JVal> &out)
    {
        ws();
        if (i >= n || s[i] != '{') return false;
        i++;
        ws();
        if (i < n && s[i] == '}') {
            i++;
            return true;
        }
        for (;;) {
            ws();
            std::string key;
            if (!str(key)) return false;
            ws();
            if (i >= n || s[i] != ':') return false;
            i++;
            JVal v;
            if (!value(v)) return false;
            out[key] = v;
            ws();
            if (i < n && s[i] == ',') {
                i++;
                continue;
            }
            if (i < n && s[i] == '}') {
                i++;
                break;
            }
            return false;
        }
        ws();
        return i == n;
    }
};

}  // namespace

extern "C" int icm_params_parse_string(icy_SimParams *p, const char *json, char *raw_points, size_t cap)
{
    if (!p || !json) return icm::fail(ICM_ERR_ARG, "icm_params_parse_string: null argument");
    Reader r{json, 0, std::strlen(json), {}};
    std::map<std::string, JVal> doc;
    if (!r.object(doc))
        return icm::fail(ICM_ERR_PARSE, "configuration file is not JSON" + (r.err.empty() ? std::string() : ": " + r.err));

    auto getd = [&](const char *k, double &dst) -> bool {
        auto it = doc.find(k);
        if (it == doc.end()) return true;
        if (it->second.kind == JVal::STR) return false;
        dst = it->second.num;
        return true;
    };
    auto geti = [&](const char *k, int &dst) -> bool {
        auto it = doc.find(k);
        if (it == doc.end()) return true;
        if (it->second.kind == JVal::STR || !it->second.is_int) return false;
        dst = (int)it->second.num;
        return true;
    };
    bool ok = true;
    ok &= getd("InitialTimeStep", p->InitialTimeStep);
    ok &= getd("YoungsModulus", p->YoungsModulus);
    ok &= geti("GridX", p->GridX);
    ok &= geti("GridY", p->GridY);
    ok &= getd("GridXDimension", p->GridXDimension);
    ok &= getd("ParticleViewSize", p->ParticleViewSize);
    ok &= getd("SimulationEndTime", p->SimulationEndTime);
    ok &= getd("PoissonsRatio", p->PoissonsRatio);
    ok &= getd("Gravity", p->Gravity);
    ok &= getd("Density", p->Density);
    ok &= getd("IndDiameter", p->IndDiameter);
    ok &= getd("IndVelocity", p->IndVelocity);
    ok &= getd("IndDepth", p->IndDepth);
    ok &= getd("IceCompressiveStrength", p->IceCompressiveStrength);
    ok &= getd("IceTensileStrength", p->IceTensileStrength);
    ok &= getd("IceShearStrength", p->IceShearStrength);
    double phi = 0;
    bool has_phi = doc.count("DP_phi") > 0;
    ok &= getd("DP_phi", phi);
    if (has_phi) p->DP_tan_phi = std::tan(phi * ICM_PI / 180);
    ok &= getd("DP_threshold_p", p->DP_threshold_p);
    ok &= getd("GrainVariability", p->GrainVariability);
    ok &= geti("UseWarpLevelReduction", p->UseWarpLevelReduction);
    ok &= geti("tpb_P2G", p->tpb_P2G);
    ok &= geti("tpb_Upd", p->tpb_Upd);
    ok &= geti("tpb_G2P", p->tpb_G2P);
    ok &= geti("SortPointsByGridCell", p->SortPointsByGridCell);
    if (!ok) return icm::fail(ICM_ERR_PARSE, "configuration value of the wrong type");
    if (p->GridX <= 0 || p->GridY <= 0 || !(p->InitialTimeStep > 0) || !(p->GridXDimension > 0))
        return icm::fail(ICM_ERR_PARSE, "configuration: grid size, dimension and time step must be positive");

    icm_params_compute_camclay(p);
    icm_params_compute_helpers(p);

    auto it = doc.find("InputRawPoints");
    if (it == doc.end() || it->second.kind != JVal::STR)
        return icm::fail(ICM_ERR_PARSE, "config parameter missing: InputRawPoints");
    if (raw_points && cap) {
        std::snprintf(raw_points, cap, "%s", it->second.str.c_str());
    }
    return ICM_OK;
}

extern "C" int icm_params_parse_file(icy_SimParams *p, const char *path, char *raw_points, size_t cap)
{
    if (!p || !path) return icm::fail(ICM_ERR_ARG, "icm_params_parse_file: null argument");
    std::ifstream f(path, std::ios::binary);
    if (!f) return icm::fail(ICM_ERR_IO, std::string("configuration file is not found: ") + path);
    std::stringstream ss;
    ss << f.rdbuf();
    std::string text = ss.str();
    return icm_params_parse_string(p, text.c_str(), raw_points, cap);
}
