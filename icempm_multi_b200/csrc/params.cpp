// params.cpp -- SimParams defaults, derived constants and the JSON reader.
//
// The reference keeps its parameters in icy::SimParams and fills it from a
// JSON file through rapidjson (simulation/parameters_sim.cpp:5-165).  This
// file gives the same results through the C-ABI struct icy_sim_params, with
// a small strict JSON reader written for this library (objects, arrays,
// strings, numbers, true/false/null; no comments), which is all the
// reference's configuration files use.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

#include "../../include/icempm.h"

namespace {

constexpr double kPi = 3.14159265358979323846;  // SimParams::pi

// ---- minimal strict JSON reader: top-level object of scalar members ----
struct JsonValue {
    enum Kind { Number, String, Bool, Null, Compound } kind = Null;
    double num = 0;
    std::string str;
};

class JsonReader {
public:
    explicit JsonReader(const char *s) : p_(s) {}
    // Parses a whole document that must be an object.  Members keep their
    // first occurrence, as rapidjson's FindMember does.
    bool parse_object(std::map<std::string, JsonValue> &out) {
        ws();
        if (*p_ != '{') return false;
        if (!object(&out)) return false;
        ws();
        return *p_ == 0;
    }

private:
    const char *p_;
    void ws() { while (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r') p_++; }
    bool lit(const char *w) {
        size_t n = std::strlen(w);
        if (std::strncmp(p_, w, n) != 0) return false;
        p_ += n;
        return true;
    }
    bool string(std::string *out) {
        if (*p_ != '"') return false;
        p_++;
        std::string s;
        while (*p_ && *p_ != '"') {
            if ((unsigned char)*p_ < 0x20) return false;
            if (*p_ == '\\') {
                p_++;
                switch (*p_) {
                case '"': s += '"'; break;
                case '\\': s += '\\'; break;
                case '/': s += '/'; break;
                case 'b': s += '\b'; break;
                case 'f': s += '\f'; break;
                case 'n': s += '\n'; break;
                case 'r': s += '\r'; break;
                case 't': s += '\t'; break;
                case 'u': {
                    unsigned v = 0;
                    for (int k = 1; k <= 4; k++) {
                        char c = p_[k];
                        v <<= 4;
                        if (c >= '0' && c <= '9') v |= c - '0';
                        else if (c >= 'a' && c <= 'f') v |= c - 'a' + 10;
                        else if (c >= 'A' && c <= 'F') v |= c - 'A' + 10;
                        else return false;
                    }
                    p_ += 4;
                    if (v < 0x80) s += (char)v;
                    else if (v < 0x800) { s += (char)(0xC0 | (v >> 6)); s += (char)(0x80 | (v & 0x3F)); }
                    else { s += (char)(0xE0 | (v >> 12)); s += (char)(0x80 | ((v >> 6) & 0x3F)); s += (char)(0x80 | (v & 0x3F)); }
                    break;
                }
                default: return false;
                }
                p_++;
            } else {
                s += *p_++;
            }
        }
        if (*p_ != '"') return false;
        p_++;
        if (out) *out = s;
        return true;
    }
    bool number(double *out) {
        const char *b = p_;
        if (*p_ == '-') p_++;
        if (*p_ == '0') p_++;
        else if (*p_ >= '1' && *p_ <= '9') { while (*p_ >= '0' && *p_ <= '9') p_++; }
        else return false;
        if (*p_ == '.') { p_++; if (!(*p_ >= '0' && *p_ <= '9')) return false; while (*p_ >= '0' && *p_ <= '9') p_++; }
        if (*p_ == 'e' || *p_ == 'E') {
            p_++;
            if (*p_ == '+' || *p_ == '-') p_++;
            if (!(*p_ >= '0' && *p_ <= '9')) return false;
            while (*p_ >= '0' && *p_ <= '9') p_++;
        }
        // strtod is correctly rounded, as rapidjson's full-precision parse
        *out = std::strtod(std::string(b, p_ - b).c_str(), nullptr);
        return true;
    }
    bool value(JsonValue *v) {
        ws();
        JsonValue tmp;
        if (*p_ == '"') { tmp.kind = JsonValue::String; if (!string(&tmp.str)) return false; }
        else if (*p_ == '{') { tmp.kind = JsonValue::Compound; if (!object(nullptr)) return false; }
        else if (*p_ == '[') { tmp.kind = JsonValue::Compound; if (!array()) return false; }
        else if (lit("true")) { tmp.kind = JsonValue::Bool; tmp.num = 1; }
        else if (lit("false")) { tmp.kind = JsonValue::Bool; tmp.num = 0; }
        else if (lit("null")) { tmp.kind = JsonValue::Null; }
        else { tmp.kind = JsonValue::Number; if (!number(&tmp.num)) return false; }
        if (v) *v = tmp;
        return true;
    }
    bool array() {
        p_++;  // '['
        ws();
        if (*p_ == ']') { p_++; return true; }
        for (;;) {
            if (!value(nullptr)) return false;
            ws();
            if (*p_ == ',') { p_++; continue; }
            if (*p_ == ']') { p_++; return true; }
            return false;
        }
    }
    bool object(std::map<std::string, JsonValue> *out) {
        p_++;  // '{'
        ws();
        if (*p_ == '}') { p_++; return true; }
        for (;;) {
            ws();
            std::string key;
            if (!string(&key)) return false;
            ws();
            if (*p_ != ':') return false;
            p_++;
            JsonValue v;
            if (!value(&v)) return false;
            if (out && out->find(key) == out->end()) (*out)[key] = v;
            ws();
            if (*p_ == ',') { p_++; continue; }
            if (*p_ == '}') { p_++; return true; }
            return false;
        }
    }
};

}  // namespace

extern "C" {

void icy_params_compute_lame(icy_sim_params *p)
{
    p->lambda = p->YoungsModulus * p->PoissonsRatio / ((1 + p->PoissonsRatio) * (1 - 2 * p->PoissonsRatio));
    p->mu = p->YoungsModulus / (2 * (1 + p->PoissonsRatio));
    p->kappa = p->mu * 2. / 3. + p->lambda;
}

void icy_params_compute_camclay(icy_sim_params *p)
{
    icy_params_compute_lame(p);
    p->NACC_beta = p->IceTensileStrength / p->IceCompressiveStrength;
    const double beta = p->NACC_beta, q = p->IceShearStrength, p0 = p->IceCompressiveStrength;
    p->NACC_M = (2 * q * std::sqrt(1 + 2 * beta)) / (p0 * (1 + beta));
    p->NACC_Msq = p->NACC_M * p->NACC_M;
}

void icy_params_compute_helpers(icy_sim_params *p)
{
    p->ParticleMass = p->ParticleVolume * p->Density;
    p->WaterParticleMass = p->ParticleVolume * p->WaterDensity;
    p->UpdateEveryNthStep = (int)(1.f / (200 * p->InitialTimeStep));
    p->cellsize = p->GridXDimension / p->GridXTotal;
    p->cellsize_inv = 1. / p->cellsize;
    p->Dp_inv = 4. / (p->cellsize * p->cellsize);
    p->IndRSq = p->IndDiameter * p->IndDiameter / 4.;
    p->dt_vol_Dpinv = p->InitialTimeStep * p->ParticleVolume * p->Dp_inv;
    p->dt_Gravity = p->InitialTimeStep * p->Gravity;
    p->vmax = 0.5 * p->cellsize / p->InitialTimeStep;
    p->vmax_squared = p->vmax * p->vmax;
    p->VectorCapacity_transfer = p->nPartitions
        ? (int)(p->nPtsTotal / p->nPartitions * p->PointsTransferBufferFraction) : 0;
    p->gbOffset = p->GridY * p->GridHaloSize;
}

void icy_params_reset(icy_sim_params *p)
{
    std::memset(p, 0, sizeof(*p));
    p->nPtsTotal = 0;
    p->n_indenter_subdivisions = 100;
    p->InitialTimeStep = 3.e-5;
    p->YoungsModulus = 5.e8;
    p->GridXTotal = 128;
    p->GridY = 55;
    p->ParticleViewSize = 2.5f;
    p->GridXDimension = 3.33;
    p->SimulationEndTime = 12;
    p->PoissonsRatio = 0.3;
    p->Gravity = 9.81;
    p->Density = 916;
    p->WaterDensity = 1000;
    p->IndDiameter = 0.324;
    p->IndVelocity = 0.2;
    p->IndDepth = 0.25;
    p->SimulationStep = 0;
    p->SimulationTime = 0;
    p->IceCompressiveStrength = 100e6;
    p->IceTensileStrength = 10e6;
    p->IceShearStrength = 6e6;
    p->IceTensileStrength2 = 5e6;
    p->DP_tan_phi = std::tan(30 * kPi / 180.);
    p->DP_threshold_p = 1e3;
    p->tpb_P2G = 256;
    p->tpb_Upd = 512;
    p->tpb_G2P = 128;
    p->indenter_x = p->indenter_x_initial = p->indenter_y = p->indenter_y_initial = 0;
    p->SetupType = 0;
    p->GrainVariability = 0.50;
    p->GridHaloSize = 5;
    p->ExtraSpaceForIncomingPoints = 0.2;
    p->PointsTransferBufferFraction = 0.05;
    p->nPartitions = 3;
    p->RebalanceThresholdFreeSpaceRemaining = 0.15;
    p->RebalanceThresholdDisabledPercentage = 0.01;
    p->PointTransferFrequency = 2;
    icy_params_compute_lame(p);
    icy_params_compute_camclay(p);
    icy_params_compute_helpers(p);
}

int icy_params_parse_json(icy_sim_params *p, const char *json_text, char *raw_points, size_t cap)
{
    if (!p || !json_text) return ICY_ERR_INVALID_ARGUMENT;
    std::map<std::string, JsonValue> doc;
    JsonReader rd(json_text);
    if (!rd.parse_object(doc)) return ICY_ERR_JSON;
    auto num = [&](const char *k, double *dst) {
        auto it = doc.find(k);
        if (it != doc.end() && it->second.kind == JsonValue::Number) *dst = it->second.num;
    };
    auto inum = [&](const char *k, int *dst) {
        auto it = doc.find(k);
        if (it != doc.end() && it->second.kind == JsonValue::Number) *dst = (int)it->second.num;
    };
    // the keys of simulation/parameters_sim.cpp:77-107, in the same order
    inum("SetupType", &p->SetupType);
    num("InitialTimeStep", &p->InitialTimeStep);
    num("YoungsModulus", &p->YoungsModulus);
    inum("GridX", &p->GridXTotal);
    inum("GridY", &p->GridY);
    num("GridXDimension", &p->GridXDimension);
    num("ParticleViewSize", &p->ParticleViewSize);
    num("SimulationEndTime", &p->SimulationEndTime);
    num("PoissonsRatio", &p->PoissonsRatio);
    num("Gravity", &p->Gravity);
    num("Density", &p->Density);
    num("IndDiameter", &p->IndDiameter);
    num("IndVelocity", &p->IndVelocity);
    num("IndDepth", &p->IndDepth);
    num("IceCompressiveStrength", &p->IceCompressiveStrength);
    num("IceTensileStrength", &p->IceTensileStrength);
    num("IceTensileStrength2", &p->IceTensileStrength2);
    num("IceShearStrength", &p->IceShearStrength);
    {
        double phi = 0;
        auto it = doc.find("DP_phi");
        if (it != doc.end() && it->second.kind == JsonValue::Number) {
            phi = it->second.num;
            p->DP_tan_phi = std::tan(phi * kPi / 180);
        }
    }
    num("DP_threshold_p", &p->DP_threshold_p);
    num("GrainVariability", &p->GrainVariability);
    inum("tpb_P2G", &p->tpb_P2G);
    inum("tpb_Upd", &p->tpb_Upd);
    inum("tpb_G2P", &p->tpb_G2P);
    inum("GridHaloSize", &p->GridHaloSize);
    inum("nPartitions", &p->nPartitions);
    num("ExtraSpaceForIncomingPoints", &p->ExtraSpaceForIncomingPoints);
    icy_params_compute_camclay(p);
    icy_params_compute_helpers(p);
    auto it = doc.find("InputRawPoints");
    if (it == doc.end() || it->second.kind != JsonValue::String) return ICY_ERR_CONFIG_MISSING;
    if (raw_points && cap) {
        std::strncpy(raw_points, it->second.str.c_str(), cap - 1);
        raw_points[cap - 1] = 0;
    }
    return ICY_OK;
}

int icy_params_parse_file(icy_sim_params *p, const char *path, char *raw_points, size_t cap)
{
    if (!path) return ICY_ERR_INVALID_ARGUMENT;
    std::ifstream f(path, std::ios::binary);
    if (!f) return ICY_ERR_FILE;
    std::stringstream ss;
    ss << f.rdbuf();
    return icy_params_parse_json(p, ss.str().c_str(), raw_points, cap);
}

}  // extern "C"
