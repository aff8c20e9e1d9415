// hidem_b200.hpp — header-only C++ adapter with the shape of the reference's HiDEMLib
// timestep surface (HiDEMLib/HiDEMLib.h:256-530) over the C ABI of hidem_b200.h.
//
// The default functors of the reference (HiDEMDefNeighForceFunc, HiDEMDefLinkForceFunc,
// HiDEMDefLinkBreakFunc, HiDEM/Common/HiDEMDefaultFunctions.h) and the sample integrate
// step are built into the library; their parameters come from the run config in
// hidem_params. computePartForce / linkUpdate therefore take no functor objects: a
// caller that needs a different functor keeps the reference's templated path.
// Errors throw hidem::Error (status + hidem_last_error text) instead of exit(1).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>

#include "hidem_b200.h"

namespace hidem {

struct Error : std::runtime_error {
    hidem_status status;
    Error(hidem_status s, const std::string &what) : std::runtime_error(what), status(s) {}
};

// The default functors' parameters, constructed as a caller's main constructs the
// reference's functors (HiDEM/Common/HiDEMDefaultFunctions.h); passing them to
// computePartForce / linkUpdate makes the library use them (hidem_set_functor_params).
struct NeighForceFunc {  // HiDEMDefNeighForceFunc
    double invDt, attractDistance, attractScaleForce, damping, dampingRotation, scaleE;
};
struct LinkForceFunc {  // HiDEMDefLinkForceFunc
    double invDt, damping, dampingRotation, E, W2, W4, G;
};
struct LinkBreakFunc {  // HiDEMDefLinkBreakFunc
    double bendBreak, maxLoad;
};

class HiDEMLibB200 {
public:
    explicit HiDEMLibB200(const hidem_params &p, int device = 0) : params_(p) {
        hidem_status s = hidem_create(&p, device, &ctx_);
        if (s != HIDEM_OK) throw Error(s, hidem_create_error());
    }
    ~HiDEMLibB200() { hidem_destroy(ctx_); }
    HiDEMLibB200(const HiDEMLibB200 &) = delete;
    HiDEMLibB200 &operator=(const HiDEMLibB200 &) = delete;

    // ParticleDataHandler::appendInitParticles / LinkDataHandler::appendInitLinks
    void setParticles(const hidem_particle_soa &p, int64_t n) { check(hidem_set_particles(ctx_, &p, n)); }
    void setLinks(const hidem_link_soa &l, int64_t L) { check(hidem_set_links(ctx_, &l, L)); }
    void setTimestep(int64_t t) { check(hidem_set_timestep(ctx_, t)); }

    // HiDEMLib::gridService / computePartForce / applyForce / linkUpdate / finalizeTs
    void gridService() { check(hidem_grid_service(ctx_)); }
    void computePartForce() { check(hidem_compute_forces(ctx_)); }
    void computePartForce(const NeighForceFunc &n, const LinkForceFunc &l) {
        hidem_functor_params f;
        check(hidem_get_functor_params(ctx_, &f));
        f.neigh_invDt = n.invDt;
        f.neigh_attractDistance = n.attractDistance;
        f.neigh_attractScaleForce = n.attractScaleForce;
        f.neigh_damping = n.damping;
        f.neigh_dampingRotation = n.dampingRotation;
        f.neigh_scaleE = n.scaleE;
        f.link_invDt = l.invDt;
        f.link_damping = l.damping;
        f.link_dampingRotation = l.dampingRotation;
        f.link_E = l.E;
        f.link_W2 = l.W2;
        f.link_W4 = l.W4;
        f.link_G = l.G;
        check(hidem_set_functor_params(ctx_, &f));
        check(hidem_compute_forces(ctx_));
    }
    void applyForce() { check(hidem_integrate(ctx_)); }
    void linkUpdate() { check(hidem_link_update(ctx_)); }
    void linkUpdate(const LinkBreakFunc &b) {
        hidem_functor_params f;
        check(hidem_get_functor_params(ctx_, &f));
        f.break_bendBreak = b.bendBreak;
        f.break_maxLoad = b.maxLoad;
        check(hidem_set_functor_params(ctx_, &f));
        check(hidem_link_update(ctx_));
    }
    void finalizeTs() { check(hidem_finalize_ts(ctx_)); }
    // n whole timesteps of the sample main loop, one fused kernel per step
    void step(int32_t n) { check(hidem_step(ctx_, n)); }

    int64_t getCurrentTimestep() {
        hidem_stats s;
        check(hidem_get_stats(ctx_, &s));
        return s.step;
    }
    // the sample main's gate `getCurrentTimestep() * dt > breakTime` in lp precision
    bool breakActive() {
        const int64_t t = getCurrentTimestep();
        if (params_.precision == HIDEM_PREC_MIXED)
            return (float)((float)t * (float)params_.dt) > (float)params_.breakTime;
        return (double)t * params_.dt > params_.breakTime;
    }

    void getParticles(hidem_particle_soa &out) { check(hidem_get_particles(ctx_, &out)); }
    void getLinks(hidem_link_soa &out) { check(hidem_get_links(ctx_, &out)); }
    void getForces(void *force[6]) { check(hidem_get_forces(ctx_, force)); }
    hidem_stats getStats() {
        hidem_stats s;
        check(hidem_get_stats(ctx_, &s));
        return s;
    }
    void synchronize() { check(hidem_synchronize(ctx_)); }
    hidem_ctx *handle() { return ctx_; }

    // HiDEMH5Checkpoint write / restart (HiDEMLib/HiDEMH5Checkpoint.h:24-50)
    void writeCheckpoint(const std::string &path) { check(hidem_checkpoint_write(ctx_, path.c_str())); }
    void readCheckpoint(const std::string &path) { check(hidem_checkpoint_read(ctx_, path.c_str())); }

    // GlacierDem bed / friction maps (InputBed) and ExternalForces maps; nullptr removes them
    void setBedMaps(const hidem_map2d *bed, const hidem_map2d *friction) {
        check(hidem_set_bed_maps(ctx_, bed, friction));
    }
    void setExternalForceMaps(const hidem_map2d maps[6]) { check(hidem_set_external_force_maps(ctx_, maps)); }

    // CollisionMesh of the MeshConstrainedDem sample: generateAccel, face forces, zeroForce
    void setCollisionMesh(const hidem_mesh *mesh) { check(hidem_set_collision_mesh(ctx_, mesh)); }
    void getMeshFaceForces(void *x, void *y, void *z) { check(hidem_get_mesh_face_forces(ctx_, x, y, z)); }
    void zeroMeshForces() { check(hidem_zero_mesh_face_forces(ctx_)); }

    // kinetic energy of the current state (translational, rotational, largest speed)
    void kineticEnergy(double &translational, double &rotational, double &maxSpeed) {
        check(hidem_kinetic_energy(ctx_, &translational, &rotational, &maxSpeed));
    }
    // step kernel (HIDEM_STEP_KERNEL_*; AUTO times the candidates on the first steps)
    void setStepKernel(int32_t kernel) { check(hidem_set_step_kernel(ctx_, kernel)); }
    void setChecks(int32_t flags) { check(hidem_set_checks(ctx_, flags)); }
    int32_t stepKernel() { return hidem_get_step_kernel(ctx_); }

    // the context's device arrays, for hidem_b200_iterate.cuh (take it again after a
    // call that rebuilds or steps)
    hidem_device_view deviceView() {
        hidem_device_view v;
        check(hidem_get_device_view(ctx_, &v));
        return v;
    }
    // computePartForce with the halo send records written by the force pass (slab ranks)
    void computePartForcePacked(void *deviceSendBuffer) {
        check(hidem_compute_forces_packed(ctx_, deviceSendBuffer));
    }

private:
    void check(hidem_status s) {
        if (s != HIDEM_OK) throw Error(s, hidem_last_error(ctx_));
    }
    hidem_params params_;
    hidem_ctx *ctx_ = nullptr;
};

}  // namespace hidem
