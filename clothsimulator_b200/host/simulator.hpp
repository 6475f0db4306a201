// Host-side mirror of the reference's scene interfaces for the `--gpu` path: Simulator, Cloth,
// Material, Handle, Wind, Magic, Transformation and Mesh, reading the same scene JSON keys
// and OBJ dialect, and stepping every cloth through the C ABI (include/clothstep.h).
//
// Only the headless modes exist (simulate_offline, resume_offline); the interactive OpenGL
// modes (simulate, resume, replay) are unavailable on a machine without a graphics stack.
// Collision, remeshing, separation and obstacles are outside the implicit step and are not
// provided: a scene that enables them is rejected with a clear error.
#ifndef CLOTHSIM_HOST_SIMULATOR_HPP
#define CLOTHSIM_HOST_SIMULATOR_HPP

#include <array>
#include <string>
#include <vector>

#include "../../include/clothstep.h"
#include "json.hpp"

namespace clothsim {

struct Vec3 {
    float x = 0, y = 0, z = 0;
};

// Transformation.cu:8-13, 78-87 and Quaternion.cu:7-15, 76-78.
class Transformation {
public:
    explicit Transformation(const Json& json);
    Vec3 applyToPoint(const Vec3& p) const;
    Vec3 applyToVector(const Vec3& v) const;
    void applyToUV(float u[2]) const;
    // the 8 values the C ABI takes (cs_step_params.transformations): scaling, translation (3),
    // rotation quaternion (s, x, y, z)
    void raw(float out[CS_TRANSFORM_FLOATS]) const;
    // applyToPoint of a transformation given by those 8 values
    static Vec3 applyRaw(const float T[CS_TRANSFORM_FLOATS], const Vec3& p);

private:
    float scaling_ = 1.0f;
    Vec3 translation_;
    float qs_ = 1.0f;  // quaternion scalar part
    Vec3 qv_;          // quaternion vector part
    Vec3 rotate(const Vec3& x) const;
};

// Motion.cu:3-72: keyframes ("time", "transform") with a keyframe of the identity at time 0
// added when the first is later, central-difference tangents (zero at the ends), and per segment
// the cubic a s^3 + b s^2 + c s + d in Transformation arithmetic (Transformation.cu:22-69,
// Quaternion.cu:23-63).  The segment index only advances, as the reference's does.
class Motion {
public:
    using T8 = std::array<float, CS_TRANSFORM_FLOATS>;
    explicit Motion(const Json& keyframes);
    T8 transformAt(float time);  // Motion::computeTransformation (Motion.cu:57-72)

private:
    std::vector<float> t_;
    std::vector<T8> x_, v_;
    T8 a_{}, b_{}, c_{}, d_{};
    int index_ = 0, n_ = 0;
    void coefficients();  // Motion::updateCoefficients (Motion.cu:48-55)
};

// Wind.cu:3-7
struct Wind {
    float density = 1.0f, drag = 0.0f;
    Vec3 velocity;
    explicit Wind(const Json& json);
};

// Magic.cu:5-17
struct Magic {
    float handleStiffness = 1e3f, collisionStiffness = 1e9f, repulsionThickness = 1e-3f, collisionThickness = 1e-4f;
    explicit Magic(const Json& json);
};

// Material.cu:3-41: the data file plus the cloth's multipliers.
class Material {
public:
    explicit Material(const Json& json);
    const cs_material_desc& desc() const { return desc_; }

private:
    cs_material_desc desc_{};
};

// Handle.cuh:9-16 (node index, motion index, target position).
struct Handle {
    int node = 0;
    int motion = -1;
    Vec3 position;
};

// Mesh::load / Mesh::save (Mesh.cu:306-507), CPU branch: nodes (x, v), uv vertices, and
// polygon faces triangulated by the fan with the largest minimum angle (Mesh.cu:27-54).
class Mesh {
public:
    void load(const std::string& path, const Transformation& transformation);
    void save(const std::string& path) const;
    std::vector<float> x, v, u;        // 3N, 3N, 2U
    std::vector<int32_t> fx, fu;       // 3F, 3F
    int nodes() const { return (int)x.size() / 3; }
    int vertices() const { return (int)u.size() / 2; }
    int faces() const { return (int)fx.size() / 3; }
};

// Cloth.cu:3-23 (constructor), 653-664 (addHandles), 865-887 (save).
class Cloth {
public:
    Cloth(const Json& json, const Wind& sceneWind);
    void addHandles(const std::vector<int>& nodeIndices, int motionIndex);
    Mesh& getMesh() { return mesh_; }
    const Material& material() const { return material_; }
    const std::vector<Handle>& handles() const { return handles_; }
    const Wind& wind() const { return wind_; }
    void save(const std::string& path, Json& json) const;

private:
    Mesh mesh_;
    Material material_;
    Wind wind_;
    std::vector<Handle> handles_;
};

struct SolverOptions {
    double tol = 1e-6;
    int maxIters = 2000;
    int precision = CS_PREC_MIXED;
    int warmStart = CS_WARM_PREVIOUS;
    int precondDegree = 3;  // strip-local Chebyshev of the cluster-resident solver (1: block-Jacobi)
    bool coarse = true;     // with it, the coarse-space correction of the cluster-resident solver
    bool warmScale = false; // the warm start replaced by its Galerkin multiple before the guard
    std::string network;  // weights for the learned warm start (CS_MLP_PARAMS floats, binary)
};

enum SimulationMode { SimulateOffline, ResumeOffline };

// Simulator.cu:3-116 (constructor), 571-600 (physicsStep), 602-684 (collisionStep), 838-897 (simulateStep),
// 950-977 (save, lastFrame, finished), 1015-1043 / 1070-1083 (offline modes).
class Simulator {
public:
    Simulator(SimulationMode mode, const std::string& path, const std::string& directory, int device = 0);
    ~Simulator();
    void start();
    void physicsStep();
    void collisionStep();
    void simulateStep();
    bool finished() const;
    void save();
    int lastFrame() const;
    int steps() const { return nSteps_; }
    int frames() const { return nFrames_; }
    std::vector<Cloth>& cloths() { return cloths_; }
    cs_step_stats lastStats() const { return stats_; }
    int lastProximities() const { return proximities_; }

private:
    SimulationMode mode_;
    std::string directory_;
    Json json_;
    float frameTime_ = 0, dt_ = 0, endTime_ = 0;
    int frameSteps_ = 1, endFrame_ = 0, nSteps_ = 0, nFrames_ = 0;
    Vec3 gravity_;
    Wind wind_;
    Magic magic_;
    float clothFriction_ = 0.6f;  // Simulator.cu:25
    int proximities_ = 0;
    cs_collision_stats collision_{};
    SolverOptions solver_;
    std::vector<Motion> motions_;   // Simulator.cu:39-80 ("motions" keyframe arrays)
    std::vector<float> transforms_; // the motions' transformations at the current step
    std::vector<Cloth> cloths_;
    cs_ctx* ctx_ = nullptr;
    cs_step_stats stats_{};
    void loadBatch(int device);
    void pullState();
    void updateTransformations();  // Simulator.cu:565-569
};

// Parses a scene without a device (counts of cloths, nodes, faces, handles); throws on error.
void describeScene(const std::string& path, long long counts[4]);

}  // namespace clothsim

#endif
