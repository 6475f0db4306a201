// Host-side scene layer for the --gpu path; see simulator.hpp.
#include "simulator.hpp"

#include <sys/stat.h>

#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <sstream>
#include <stdexcept>

namespace clothsim {

namespace {

Vec3 parseVec3(const Json& j) {
    Vec3 v;
    if (j.isNull()) return v;
    v.x = j[0].asFloat();
    v.y = j[1].asFloat();
    v.z = j[2].asFloat();
    return v;
}

float dot(const Vec3& a, const Vec3& b) {
    float s = a.x * b.x;
    s += a.y * b.y;
    s += a.z * b.z;
    return s;
}
Vec3 cross(const Vec3& a, const Vec3& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
Vec3 scale(float s, const Vec3& a) { return {s * a.x, s * a.y, s * a.z}; }
Vec3 add(const Vec3& a, const Vec3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
Vec3 sub(const Vec3& a, const Vec3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
Vec3 normalized(const Vec3& a) {
    float inv = 1.0f / std::sqrt(dot(a, a));
    return {a.x * inv, a.y * inv, a.z * inv};
}

bool exists(const std::string& p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0;
}

void makeDirs(const std::string& d) {
    std::string cur;
    std::stringstream ss(d);
    std::string part;
    if (!d.empty() && d[0] == '/') cur = "/";
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        mkdir(cur.c_str(), 0755);
    }
}

std::vector<std::string> split(const std::string& s, char c) {  // Mesh.cu:9-19
    std::vector<std::string> out;
    std::string t = s;
    size_t i;
    while ((i = t.find(c)) != std::string::npos) {
        out.push_back(t.substr(0, i));
        t.erase(0, i + 1);
    }
    out.push_back(t);
    return out;
}

float angleAt(const Vec3& x0, const Vec3& x1, const Vec3& x2) {  // Mesh.cu:21-25
    Vec3 e1 = normalized(sub(x1, x0)), e2 = normalized(sub(x2, x0));
    float c = dot(e1, e2);
    c = c < -1.0f ? -1.0f : (c > 1.0f ? 1.0f : c);
    return std::acos(c);
}

}  // namespace

// ---- Transformation -----------------------------------------------------------------------

Transformation::Transformation(const Json& json) {
    scaling_ = parseFloat(json["scale"], 1.0f);
    translation_ = parseVec3(json["translate"]);
    float r[4] = {0, 0, 0, 0};
    if (!json["rotate"].isNull())
        for (int i = 0; i < 4; i++) r[i] = json["rotate"][i].asFloat();
    const float angle = (float)(r[0] * M_PI / 180.0f);
    if (angle == 0.0f) {
        qs_ = 1.0f;
        qv_ = Vec3();
    } else {
        qs_ = std::cos(0.5f * angle);
        qv_ = scale(std::sin(0.5f * angle), normalized({r[1], r[2], r[3]}));
    }
}

Vec3 Transformation::rotate(const Vec3& x) const {
    return add(add(scale(qs_ * qs_ - dot(qv_, qv_), x), scale(2.0f * dot(qv_, x), qv_)), scale(2.0f * qs_, cross(qv_, x)));
}
Vec3 Transformation::applyToPoint(const Vec3& p) const { return add(scale(scaling_, rotate(p)), translation_); }
void Transformation::raw(float out[CS_TRANSFORM_FLOATS]) const {
    const float r[CS_TRANSFORM_FLOATS] = {scaling_, translation_.x, translation_.y, translation_.z, qs_, qv_.x, qv_.y, qv_.z};
    std::copy(r, r + CS_TRANSFORM_FLOATS, out);
}
Vec3 Transformation::applyRaw(const float T[CS_TRANSFORM_FLOATS], const Vec3& p) {
    const float qs = T[4];
    const Vec3 qv = {T[5], T[6], T[7]};
    const Vec3 r = add(add(scale(qs * qs - dot(qv, qv), p), scale(2.0f * dot(qv, p), qv)), scale(2.0f * qs, cross(qv, p)));
    return add(scale(T[0], r), {T[1], T[2], T[3]});
}

// ---- Motion ---------------------------------------------------------------------------------

namespace {
using T8 = Motion::T8;
T8 t8add(const T8& a, const T8& b) {
    T8 r;
    for (int k = 0; k < CS_TRANSFORM_FLOATS; k++) r[k] = a[k] + b[k];
    return r;
}
T8 t8sub(const T8& a, const T8& b) {
    T8 r;
    for (int k = 0; k < CS_TRANSFORM_FLOATS; k++) r[k] = a[k] - b[k];
    return r;
}
T8 t8mul(const T8& a, float s) {  // Transformation::operator*(float), Quaternion::operator*(float)
    T8 r;
    for (int k = 0; k < CS_TRANSFORM_FLOATS; k++) r[k] = a[k] * s;
    return r;
}
// Transformation::operator/(float): scaling and the quaternion's scalar part divided, translation and
// the quaternion's vector part multiplied by the reciprocal (Vector::operator/, Vector.cuh:126-132)
T8 t8div(const T8& a, float s) {
    const float inv = 1.0f / s;
    T8 r;
    for (int k = 0; k < CS_TRANSFORM_FLOATS; k++) r[k] = a[k] * inv;
    r[0] = a[0] / s;
    r[4] = a[4] / s;
    return r;
}
T8 t8identity() { return {1.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f}; }
}  // namespace

Motion::Motion(const Json& keyframes) {
    for (const Json& k : keyframes.items()) {
        t_.push_back(parseFloat(k["time"]));
        T8 x;
        Transformation(k["transform"]).raw(x.data());
        x_.push_back(x);
    }
    if (t_.empty()) throw std::runtime_error("a motion needs keyframes");
    if (t_[0] > 0) {
        t_.insert(t_.begin(), 0.0f);
        x_.insert(x_.begin(), t8identity());
    }
    n_ = (int)t_.size();
    if (n_ < 2) throw std::runtime_error("a motion needs two keyframes (one may be the time-0 identity)");
    for (int i = 1; i < n_; i++)
        if (!(t_[i] > t_[i - 1])) throw std::runtime_error("motion keyframe times must increase");
    v_.assign(n_, t8mul(t8identity(), 0.0f));
    for (int i = 1; i < n_ - 1; i++) v_[i] = t8div(t8sub(x_[i + 1], x_[i - 1]), t_[i + 1] - t_[i - 1]);
    coefficients();
}

void Motion::coefficients() {
    const float dt = t_[index_ + 1] - t_[index_];
    const T8 dx = t8sub(x_[index_ + 1], x_[index_]);
    a_ = t8sub(t8mul(t8add(v_[index_ + 1], v_[index_]), dt), t8mul(dx, 2.0f));
    b_ = t8sub(t8mul(dx, 3.0f), t8mul(t8add(v_[index_ + 1], t8mul(v_[index_], 2.0f)), dt));
    c_ = t8mul(v_[index_], dt);
    d_ = x_[index_];
}

Motion::T8 Motion::transformAt(float time) {
    bool moved = false;
    while (index_ < n_ - 1 && t_[index_ + 1] < time) {
        index_++;
        moved = true;
    }
    if (index_ == n_ - 1) return x_[n_ - 1];
    if (moved) coefficients();
    const float s = (time - t_[index_]) / (t_[index_ + 1] - t_[index_]);
    const float s2 = s * s, s3 = s * s2;
    return t8add(t8add(t8add(t8mul(a_, s3), t8mul(b_, s2)), t8mul(c_, s)), d_);
}
Vec3 Transformation::applyToVector(const Vec3& v) const { return rotate(v); }
void Transformation::applyToUV(float u[2]) const {
    u[0] *= scaling_;
    u[1] *= scaling_;
}

Wind::Wind(const Json& json) {
    density = parseFloat(json["density"], 1.0f);
    drag = parseFloat(json["drag"]);
    velocity = parseVec3(json["velocity"]);
}

Magic::Magic(const Json& json) {
    if (json.isNull()) return;
    handleStiffness = parseFloat(json["handle_stiffness"], handleStiffness);
    collisionStiffness = parseFloat(json["collision_stiffness"], collisionStiffness);
    repulsionThickness = parseFloat(json["repulsion_thickness"], repulsionThickness);
    collisionThickness = parseFloat(json["projection_thickness"], 0.1f * repulsionThickness);
}

Material::Material(const Json& json) {
    const std::string path = parseString(json["data"]);
    if (path.empty()) throw std::runtime_error("cloth materials: missing \"data\"");
    Json data = Json::parseFile(path);
    desc_.density = parseFloat(data["density"]);
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 4; j++) desc_.stretching[i][j] = data["stretching"][i][j].asFloat();
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 5; j++) desc_.bending[i][j] = data["bending"][i][j].asFloat();
    desc_.thicken = parseFloat(json["thicken"], 1.0f);
    desc_.density_mult = parseFloat(json["density_mult"], 1.0f);
    desc_.stretching_mult = parseFloat(json["stretching_mult"], 1.0f);
    desc_.bending_mult = parseFloat(json["bending_mult"], 1.0f);
}

// ---- Mesh -----------------------------------------------------------------------------------

void Mesh::load(const std::string& path, const Transformation& tr) {
    std::ifstream fin(path);
    if (!fin.is_open()) throw std::runtime_error("Failed to open mesh file: " + path);
    std::vector<Vec3> raw, xs, vs;
    std::vector<float> uv;
    fx.clear();
    fu.clear();
    std::string line;
    while (std::getline(fin, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        std::vector<std::string> s = split(line, ' ');
        if (s[0] == "v") {
            Vec3 p{std::stof(s[1]), std::stof(s[2]), std::stof(s[3])};
            raw.push_back(p);
            xs.push_back(tr.applyToPoint(p));
        } else if (s[0] == "nv") {
            vs.push_back(tr.applyToVector({std::stof(s[1]), std::stof(s[2]), std::stof(s[3])}));
        } else if (s[0] == "vt") {
            float u[2] = {std::stof(s[1]), std::stof(s[2])};
            tr.applyToUV(u);
            uv.push_back(u[0]);
            uv.push_back(u[1]);
        } else if (s[0] == "f") {
            std::vector<int> xp, up;
            for (size_t i = 1; i < s.size(); i++) {
                if (s[i].empty()) continue;
                if (line.find('/') != std::string::npos) {
                    std::vector<std::string> t = split(s[i], '/');
                    xp.push_back(std::stoi(t[0]) - 1);
                    up.push_back(std::stoi(t[1]) - 1);
                } else {
                    int xi = std::stoi(s[i]) - 1;
                    if (xi < 0 || xi >= (int)raw.size()) throw std::runtime_error(path + ": face index out of range");
                    float u[2] = {raw[xi].x, raw[xi].y};
                    tr.applyToUV(u);
                    uv.push_back(u[0]);
                    uv.push_back(u[1]);
                    xp.push_back(xi);
                    up.push_back((int)uv.size() / 2 - 1);
                }
            }
            const int n = (int)xp.size();
            if (n < 3) throw std::runtime_error(path + ": face with fewer than 3 corners");
            for (int i = 0; i < n; i++)
                if (xp[i] < 0 || xp[i] >= (int)xs.size()) throw std::runtime_error(path + ": face index out of range");
            // Mesh.cu:27-54: fan from the corner whose fan has the largest minimum angle
            float best = -std::numeric_limits<float>::infinity();
            int index = 0;
            for (int i = 0; i < n; i++) {
                float mn = std::numeric_limits<float>::infinity();
                const Vec3 x0 = xs[xp[i]];
                for (int j = 2; j < n; j++) {
                    const Vec3 x1 = xs[xp[(i + j - 1) % n]], x2 = xs[xp[(i + j) % n]];
                    mn = std::min(mn, std::min(angleAt(x0, x1, x2), std::min(angleAt(x1, x2, x0), angleAt(x2, x0, x1))));
                }
                if (mn > best) {
                    best = mn;
                    index = i;
                }
            }
            for (int i = 2; i < n; i++) {
                fx.insert(fx.end(), {xp[index], xp[(index + i - 1) % n], xp[(index + i) % n]});
                fu.insert(fu.end(), {up[index], up[(index + i - 1) % n], up[(index + i) % n]});
            }
        }
    }
    x.clear();
    v.clear();
    for (size_t i = 0; i < xs.size(); i++) {
        x.insert(x.end(), {xs[i].x, xs[i].y, xs[i].z});
        const Vec3 vi = i < vs.size() ? vs[i] : Vec3();
        v.insert(v.end(), {vi.x, vi.y, vi.z});
    }
    u = uv;
    for (int i : fu)
        if (i < 0 || i >= vertices()) throw std::runtime_error(path + ": uv index out of range");
}

void Mesh::save(const std::string& path) const {  // Mesh.cu:454-507
    std::ofstream fout(path);
    if (!fout.is_open()) throw std::runtime_error("cannot write " + path);
    fout.precision(20);
    for (int i = 0; i < nodes(); i++) {
        fout << "v " << x[3 * i] << " " << x[3 * i + 1] << " " << x[3 * i + 2] << "\n";
        fout << "nv " << v[3 * i] << " " << v[3 * i + 1] << " " << v[3 * i + 2] << "\n";
    }
    for (int i = 0; i < vertices(); i++) fout << "vt " << u[2 * i] << " " << u[2 * i + 1] << "\n";
    for (int f = 0; f < faces(); f++) {
        fout << "f";
        for (int c = 0; c < 3; c++) fout << " " << fx[3 * f + c] + 1 << "/" << fu[3 * f + c] + 1;
        fout << "\n";
    }
}

// ---- Cloth ----------------------------------------------------------------------------------

Cloth::Cloth(const Json& json, const Wind& sceneWind)
    : material_(json["materials"]), wind_(json["wind"].isNull() ? sceneWind : Wind(json["wind"])) {
    Transformation tr(json["transform"]);
    mesh_.load(parseString(json["mesh"]), tr);
}

void Cloth::addHandles(const std::vector<int>& nodeIndices, int motionIndex) {
    for (int n : nodeIndices) {
        if (n < 0 || n >= mesh_.nodes()) throw std::runtime_error("handle node " + std::to_string(n) + " out of range");
        Handle h;
        h.node = n;
        h.motion = motionIndex;
        h.position = {mesh_.x[3 * n], mesh_.x[3 * n + 1], mesh_.x[3 * n + 2]};
        handles_.push_back(h);
    }
}

void Cloth::save(const std::string& path, Json& json) const {
    json.set("mesh", Json::string(path));
    json.set("transform", Json());
    mesh_.save(path);
}

// ---- Simulator ------------------------------------------------------------------------------

static SolverOptions parseSolver(const Json& j) {
    SolverOptions o;
    if (j.isNull()) return o;
    o.tol = j["tol"].isNull() ? o.tol : j["tol"].asDouble();
    o.maxIters = parseInt(j["max_iters"], o.maxIters);
    const std::string prec = parseString(j["precision"], "mixed");
    if (prec == "mixed") o.precision = CS_PREC_MIXED;
    else if (prec == "plain") o.precision = CS_PREC_PLAIN_FP32;
    else throw std::runtime_error("solver.precision must be \"mixed\" or \"plain\"");
    const std::string warm = parseString(j["warm_start"], "previous");
    if (warm == "previous") o.warmStart = CS_WARM_PREVIOUS;
    else if (warm == "zero") o.warmStart = CS_WARM_ZERO;
    else if (warm == "learned") o.warmStart = CS_WARM_LEARNED;
    else throw std::runtime_error("solver.warm_start must be \"previous\", \"zero\" or \"learned\"");
    o.precondDegree = parseInt(j["precond_degree"], o.precondDegree);
    if (o.precondDegree < 0 || o.precondDegree > CS_PRECOND_MAX_DEGREE || (o.precondDegree > 1 && o.precondDegree % 2 == 0))
        throw std::runtime_error("solver.precond_degree must be 0, 1 or an odd degree up to 15");
    if (!j["coarse"].isNull()) o.coarse = j["coarse"].asDouble() != 0.0;
    if (!j["warm_scale"].isNull()) o.warmScale = j["warm_scale"].asDouble() != 0.0;
    o.network = parseString(j["network"]);
    if (o.warmStart == CS_WARM_LEARNED && o.network.empty())
        throw std::runtime_error("solver.warm_start \"learned\" needs solver.network (a weights file)");
    return o;
}

static void checkSupported(const Json& json) {
    if (json["motions"].isObject())
        throw std::runtime_error("\"motions\" from a motion file (.mot, Simulator.cu:43-80) are not provided: give "
                                 "keyframe arrays");
    if (!json["obstacles"].isNull() && (json["obstacles"].size() > 0 || json["obstacles"].type() == Json::String))
        throw std::runtime_error("\"obstacles\" are not provided: collisions are handled among cloths only");
    bool remeshingOff = false;
    for (const Json& d : json["disable"].items())
        if (d.type() == Json::String && d.asString() == "remeshing") remeshingOff = true;
    if (!remeshingOff) throw std::runtime_error("remeshing is not provided: add \"remeshing\" to \"disable\"");
}

void describeScene(const std::string& path, long long counts[4]) {
    Json json = Json::parseFile(path);
    checkSupported(json);
    Wind wind(json["wind"]);
    counts[0] = counts[1] = counts[2] = counts[3] = 0;
    std::vector<Cloth> cloths;
    for (const Json& c : json["cloths"].items()) cloths.emplace_back(c, wind);
    for (const Json& h : json["handles"].items()) {
        int ci = parseInt(h["cloth"]);
        if (ci < 0 || ci >= (int)cloths.size()) throw std::runtime_error("handle cloth index out of range");
        std::vector<int> nodes;
        for (const Json& n : h["nodes"].items()) nodes.push_back(n.asInt());
        const int mi = parseInt(h["motion"], -1);
        if (mi < -1 || mi >= (int)json["motions"].size()) throw std::runtime_error("handle motion index out of range");
        cloths[ci].addHandles(nodes, mi);
    }
    counts[0] = (long long)cloths.size();
    for (Cloth& c : cloths) {
        counts[1] += c.getMesh().nodes();
        counts[2] += c.getMesh().faces();
        counts[3] += (long long)c.handles().size();
    }
}

Simulator::Simulator(SimulationMode mode, const std::string& path, const std::string& directory, int device)
    : mode_(mode), directory_(directory), wind_(Json()), magic_(Json()) {
    json_ = Json::parseFile(mode == SimulateOffline ? path : directory + "/config.json");
    checkSupported(json_);
    frameTime_ = parseFloat(json_["frame_time"]);
    frameSteps_ = parseInt(json_["frame_steps"]);
    if (!(frameTime_ > 0) || frameSteps_ <= 0) throw std::runtime_error("frame_time and frame_steps must be positive");
    endTime_ = parseFloat(json_["end_time"], std::numeric_limits<float>::infinity());
    endFrame_ = parseInt(json_["end_frame"], INT_MAX);
    dt_ = frameTime_ / frameSteps_;
    gravity_ = parseVec3(json_["gravity"]);
    wind_ = Wind(json_["wind"]);
    magic_ = Magic(json_["magic"]);
    clothFriction_ = parseFloat(json_["friction"], 0.6f);  // Simulator.cu:25
    solver_ = parseSolver(json_["solver"]);
    for (const Json& m : json_["motions"].items()) motions_.emplace_back(m);
    if ((int)motions_.size() > CS_MAX_MOTIONS) throw std::runtime_error("more than CS_MAX_MOTIONS motions");
    for (const Json& c : json_["cloths"].items()) cloths_.emplace_back(c, wind_);
    if (cloths_.empty()) throw std::runtime_error("scene has no cloths");
    for (const Json& h : json_["handles"].items()) {
        int ci = parseInt(h["cloth"]);
        if (ci < 0 || ci >= (int)cloths_.size()) throw std::runtime_error("handle cloth index out of range");
        std::vector<int> nodes;
        for (const Json& n : h["nodes"].items()) nodes.push_back(n.asInt());
        const int mi = parseInt(h["motion"], -1);
        if (mi < -1 || mi >= (int)motions_.size()) throw std::runtime_error("handle motion index out of range");
        cloths_[ci].addHandles(nodes, mi);
    }
    loadBatch(device);
}

Simulator::~Simulator() {
    if (ctx_) cs_destroy(ctx_);
}

void Simulator::loadBatch(int device) {
    cs_status st = cs_create(&ctx_, device);
    if (st != CS_OK) throw std::runtime_error("no usable sm_100 CUDA device (status " + std::to_string(st) + ")");
    std::vector<cs_material_desc> mats;
    std::vector<cs_sheet_desc> sheets;
    std::vector<std::vector<int32_t>> handleNodes(cloths_.size());
    std::vector<std::vector<float>> handlePos(cloths_.size());
    for (size_t i = 0; i < cloths_.size(); i++) {
        Cloth& c = cloths_[i];
        Mesh& m = c.getMesh();
        mats.push_back(c.material().desc());
        for (const Handle& h : c.handles()) {
            handleNodes[i].push_back(h.node);
            handlePos[i].insert(handlePos[i].end(), {h.position.x, h.position.y, h.position.z});
        }
        cs_sheet_desc d{};
        d.n_nodes = m.nodes();
        d.n_verts = m.vertices();
        d.n_faces = m.faces();
        d.n_handles = (int)handleNodes[i].size();
        d.x = m.x.data();
        d.v = m.v.data();
        d.uv = m.u.data();
        d.face_nodes = m.fx.data();
        d.face_verts = m.fu.data();
        d.handle_nodes = handleNodes[i].data();
        d.handle_pos = handlePos[i].data();
        d.material = (int)i;
        d.wind_density = c.wind().density;
        d.wind_drag = c.wind().drag;
        d.wind_velocity[0] = c.wind().velocity.x;
        d.wind_velocity[1] = c.wind().velocity.y;
        d.wind_velocity[2] = c.wind().velocity.z;
        sheets.push_back(d);
    }
    st = cs_load_batch(ctx_, mats.data(), (int)mats.size(), sheets.data(), (int)sheets.size());
    if (st != CS_OK) throw std::runtime_error(std::string("cs_load_batch: ") + cs_last_error(ctx_));
    // handles that follow a motion (Simulator.cu:104-111)
    std::vector<int32_t> motion;
    bool moving = false;
    for (const Cloth& c : cloths_)
        for (const Handle& h : c.handles()) {
            motion.push_back(h.motion);
            moving |= h.motion > -1;
        }
    if (moving && cs_set_handle_motions(ctx_, motion.data(), (int)motion.size()) != CS_OK)
        throw std::runtime_error(std::string("cs_set_handle_motions: ") + cs_last_error(ctx_));
    if (solver_.warmStart == CS_WARM_LEARNED) {
        std::vector<float> w(CS_MLP_PARAMS);
        std::ifstream in(solver_.network, std::ios::binary);
        if (!in.read(reinterpret_cast<char*>(w.data()), (std::streamsize)(w.size() * sizeof(float))))
            throw std::runtime_error("cannot read network weights " + solver_.network);
        if (cs_mlp_init(ctx_, 0, 0) != CS_OK || cs_mlp_set_weights(ctx_, w.data(), CS_MLP_PARAMS) != CS_OK)
            throw std::runtime_error(std::string("network: ") + cs_last_error(ctx_));
    }
}

// Simulator.cu:571-600: proximities among the cloths' current states (findProximitiesGpu), then
// every cloth's implicit step with them, then the position update (inside cs_step).
void Simulator::physicsStep() {
    cs_detect_params dp{};
    dp.repulsion_thickness = magic_.repulsionThickness;
    dp.collision_stiffness = magic_.collisionStiffness;
    dp.friction = clothFriction_;
    dp.sheet_group = nullptr;  // the cloths of one scene interact
    if (cs_detect_proximities(ctx_, &dp, &proximities_) != CS_OK)
        throw std::runtime_error(std::string("cs_detect_proximities: ") + cs_last_error(ctx_));
    cs_step_params p{};
    p.dt = dt_;
    p.gravity[0] = gravity_.x;
    p.gravity[1] = gravity_.y;
    p.gravity[2] = gravity_.z;
    p.handle_stiffness = magic_.handleStiffness;
    p.tol = solver_.tol;
    p.max_iters = solver_.maxIters;
    p.precision = solver_.precision;
    p.precond_degree = solver_.precondDegree;
    p.coarse = solver_.coarse ? 1 : 0;
    p.warm_scale = solver_.warmScale ? 1 : 0;
    p.transformations = transforms_.empty() ? nullptr : transforms_.data();
    p.n_transformations = (int)motions_.size();
    p.warm_start = nSteps_ > 1 || mode_ == ResumeOffline ? solver_.warmStart : CS_WARM_ZERO;
    if (solver_.warmStart == CS_WARM_LEARNED) p.warm_start = CS_WARM_LEARNED;
    p.advance = 1;
    p.use_graph = 1;
    cs_status st = cs_step(ctx_, &p, &stats_);
    if (st == CS_ERR_NOT_CONVERGED)
        std::cerr << "warning: " << cs_last_error(ctx_) << std::endl;
    else if (st != CS_OK)
        throw std::runtime_error(std::string("cs_step: ") + cs_last_error(ctx_));
}

// Simulator.cu:571-684: the positions cs_step produced are resolved against the impacts
// between the start and the end of the step, then v = (x - x0) / dt.
void Simulator::collisionStep() {
    cs_collision_params cp{};
    cp.thickness = magic_.collisionThickness;
    cp.dt = dt_;
    cp.sheet_group = nullptr;
    cs_status st = cs_collision_step(ctx_, &cp, &collision_);
    if (st == CS_ERR_NOT_CONVERGED) throw std::runtime_error("Collision step failed!");  // Simulator.cu:668-671
    if (st != CS_OK) throw std::runtime_error(std::string("cs_collision_step: ") + cs_last_error(ctx_));
}

void Simulator::updateTransformations() {
    const float time = nSteps_ * dt_;
    transforms_.assign(CS_TRANSFORM_FLOATS * motions_.size(), 0.0f);
    for (size_t i = 0; i < motions_.size(); i++) {
        const Motion::T8 t = motions_[i].transformAt(time);
        std::copy(t.begin(), t.end(), transforms_.begin() + CS_TRANSFORM_FLOATS * i);
    }
}

void Simulator::simulateStep() {
    if ((++nSteps_) % frameSteps_ == 0) nFrames_++;
    std::cout << "Frame [" << nFrames_ << "], Step [" << nSteps_ << "]:" << std::endl;
    updateTransformations();
    physicsStep();
    std::cout << "Physics Step: " << stats_.ms / 1000.0 << "s (" << proximities_ << " proximities, " << stats_.max_iters
              << " CG iterations, relative residual " << stats_.max_rel_residual << ")";
    collisionStep();
    std::cout << ", Collision Step: " << collision_.rounds << " rounds, " << collision_.impacts << " impacts" << std::endl;
    if (nSteps_ % frameSteps_ == 0) save();
}

bool Simulator::finished() const { return nSteps_ * dt_ >= endTime_ || nFrames_ >= endFrame_; }

void Simulator::pullState() {
    long long sizes[7];
    cs_get_sizes(ctx_, sizes);
    std::vector<float> x(3 * sizes[0]), v(3 * sizes[0]);
    if (cs_get_state(ctx_, x.data(), v.data()) != CS_OK) throw std::runtime_error(cs_last_error(ctx_));
    size_t off = 0;
    for (Cloth& c : cloths_) {
        Mesh& m = c.getMesh();
        std::copy(x.begin() + off, x.begin() + off + m.x.size(), m.x.begin());
        std::copy(v.begin() + off, v.begin() + off + m.v.size(), m.v.begin());
        off += m.x.size();
    }
}

void Simulator::save() {
    pullState();
    for (size_t i = 0; i < cloths_.size(); i++)
        cloths_[i].save(directory_ + "/frame" + std::to_string(nFrames_) + "_cloth" + std::to_string(i) + ".obj",
                        json_.at("cloths").at(i));
    std::ofstream fout(directory_ + "/config.json");
    fout << json_.dump(4) << std::endl;
}

int Simulator::lastFrame() const {
    int ans = 0;
    for (;;) {
        ans++;
        for (size_t i = 0; i < cloths_.size(); i++)
            if (!exists(directory_ + "/frame" + std::to_string(ans) + "_cloth" + std::to_string(i) + ".obj")) return ans - 1;
    }
}

void Simulator::start() {
    auto t0 = std::chrono::steady_clock::now();
    if (mode_ == SimulateOffline) {
        makeDirs(directory_);
        save();
    } else {
        nFrames_ = lastFrame();
        nSteps_ = nFrames_ * frameSteps_;
    }
    while (!finished()) simulateStep();
    auto t1 = std::chrono::steady_clock::now();
    std::cout << "Total time: " << std::chrono::duration<double>(t1 - t0).count() << "s" << std::endl;
}

}  // namespace clothsim

// ---- C entry points of the host layer -------------------------------------------------------

static std::string g_sim_error;

extern "C" const char* cs_sim_last_error() { return g_sim_error.c_str(); }

// The host layer's Transformation(json).applyToPoint and Motion(keyframes).computeTransformation
// applied to points, for checking them against the reference's (json_text: a "transform" object,
// or a "motions" keyframe array).  Return 0, or CS_ERR_INVALID_ARG with cs_sim_last_error.
extern "C" int cs_transform_points(const char* json_text, int n, const double* p, double* out) {
    try {
        clothsim::Transformation t(clothsim::Json::parse(json_text));
        for (int i = 0; i < n; i++) {
            const clothsim::Vec3 q = t.applyToPoint({(float)p[3 * i], (float)p[3 * i + 1], (float)p[3 * i + 2]});
            out[3 * i] = q.x;
            out[3 * i + 1] = q.y;
            out[3 * i + 2] = q.z;
        }
        return 0;
    } catch (const std::exception& e) {
        g_sim_error = e.what();
        return CS_ERR_INVALID_ARG;
    }
}

extern "C" int cs_motion_points(const char* json_text, int n_times, const double* times, int n, const double* p,
                                double* out, float* transforms) {
    try {
        clothsim::Motion m(clothsim::Json::parse(json_text));
        for (int k = 0; k < n_times; k++) {
            const clothsim::Motion::T8 t = m.transformAt((float)times[k]);
            if (transforms) std::copy(t.begin(), t.end(), transforms + CS_TRANSFORM_FLOATS * k);
            for (int i = 0; i < n; i++) {
                const clothsim::Vec3 q = clothsim::Transformation::applyRaw(
                    t.data(), {(float)p[3 * i], (float)p[3 * i + 1], (float)p[3 * i + 2]});
                out[3 * (k * n + i)] = q.x;
                out[3 * (k * n + i) + 1] = q.y;
                out[3 * (k * n + i) + 2] = q.z;
            }
        }
        return 0;
    } catch (const std::exception& e) {
        g_sim_error = e.what();
        return CS_ERR_INVALID_ARG;
    }
}

// Reads an OBJ mesh as a cloth's mesh is read (Mesh::load, Mesh.cu:306-452: v, nv, vt, f with
// a/b or plain indices, polygons fan-triangulated) and writes it as a frame (Mesh::save,
// Mesh.cu:454-507).  Return 0, or CS_ERR_INVALID_ARG with cs_sim_last_error.
extern "C" int cs_mesh_rewrite(const char* in_path, const char* out_path) {
    try {
        clothsim::Mesh m;
        m.load(in_path, clothsim::Transformation(clothsim::Json()));
        m.save(out_path);
        return 0;
    } catch (const std::exception& e) {
        g_sim_error = e.what();
        return CS_ERR_INVALID_ARG;
    }
}

extern "C" int cs_scene_describe(const char* path, long long* counts) {
    try {
        clothsim::describeScene(path, counts);
        return CS_OK;
    } catch (const std::exception& e) {
        g_sim_error = e.what();
        return CS_ERR_INVALID_ARG;
    }
}

extern "C" int cs_sim_run(const char* mode, const char* path, const char* dir, int device, int* steps) {
    try {
        std::string m = mode ? mode : "";
        if (m == "simulate" || m == "resume" || m == "replay") {
            g_sim_error = "mode \"" + m + "\" needs OpenGL/GLFW, unavailable on this machine; use " + m + "_offline";
            return CS_ERR_INVALID_ARG;
        }
        clothsim::SimulationMode sm;
        if (m == "simulate_offline") sm = clothsim::SimulateOffline;
        else if (m == "resume_offline") sm = clothsim::ResumeOffline;
        else {
            g_sim_error = "mode should be one of simulate_offline/resume_offline";
            return CS_ERR_INVALID_ARG;
        }
        clothsim::Simulator s(sm, path ? path : "", dir ? dir : "", device);
        s.start();
        if (steps) *steps = s.steps();
        return CS_OK;
    } catch (const std::exception& e) {
        g_sim_error = e.what();
        return g_sim_error.find("sm_100") != std::string::npos ? CS_ERR_NO_DEVICE : CS_ERR_INVALID_ARG;
    }
}
