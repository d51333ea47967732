/*
 * macnbflip3_b200 -- Shiokaze FLIP module (FLIP=macnbflip3_b200) whose splat
 * runs on a B200.
 *
 * It is the reference's narrow-band FLIP, macnbflip3 (src/flip/macnbflip3.cpp),
 * compiled into this module from the reference tree where it lies, with one
 * method replaced: splat(time, mass_and_momentum)
 * (macflip3_interface::splat, include/shiokaze/flip/macflip3_interface.h:79;
 * macnbflip3.cpp:103-148). The override hands the module's own particle
 * vector to shkz_b200_splat_host in place (stride sizeof(Particle), the
 * fields' offsets) and fills mass_and_momentum from the splat grid it
 * returns: the faces with non-zero mass, each with its mass and momentum,
 * bit-identical to the reference's. Advection, seeding, bullets, correction
 * and the particle update stay the reference's code.
 *
 * The reference's own module entry points in macnbflip3.cpp are renamed
 * while it is compiled here, so that this file's create_instance() is the
 * one the module loader finds.
 *
 * Errors never throw: a failed splat is reported on the console and leaves
 * mass_and_momentum empty (the liquid solver then keeps its grid velocity).
 * With B200.Strict=Yes a failure ends the program (exit status 1).
 */
#define create_instance shkz_macnbflip3_reference_create_instance
#define license shkz_macnbflip3_reference_license
#include "macnbflip3.cpp"
#undef create_instance
#undef license
#include <shiokaze/core/console.h>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "shkz_b200.h"
//
SHKZ_USING_NAMESPACE
//
class macnbflip3_b200 : public macnbflip3 {
protected:
	//
	LONG_NAME("MAC Narrowband FLIP 3D (B200 splat)")
	//
	virtual ~macnbflip3_b200() {
		if( m_ctx ) shkz_b200_destroy(m_ctx);
	}
	//
	virtual void configure( configuration &config ) override {
		macnbflip3::configure(config);
		config.get_bool("B200.Strict",m_strict,"End the program when the GPU splat fails");
		config.get_integer("B200.Device",m_device,"CUDA device of the splat");
	}
	//
	bool fail( const char *what, int rc ) const {
		console::dump( "%s failed: %s (%s)\n", what, shkz_b200_errstr(rc), m_ctx ? shkz_b200_last_error(m_ctx) : "");
		if( m_strict ) std::exit(1);
		return false;
	}
	//
	virtual void splat( double time, macarray3<macflip3_interface::mass_momentum3> &mass_and_momentum ) const override {
		//
		scoped_timer timer(this);
		mass_and_momentum.clear();
		if( m_particles.empty()) return;
		timer.tick(); console::dump( "Splatting momentum (B200)...");
		if( ! m_ctx ) {
			shkz_b200_config cfg;
			shkz_b200_default_config(&cfg);
			cfg.device = m_device;
			int rc = shkz_b200_create(&m_ctx,&cfg);
			if( rc ) { fail("shkz_b200_create",rc); return; }
		}
		const shape3 s = m_shape;
		// the splat grid only (no velocity: the entry point then forms no
		// combined velocity and copies no velocity grid)
		std::vector<float> mass[3], momentum[3];
		std::vector<uint8_t> splat_active[3];
		shkz_b200_splat_args a;
		std::memset(&a,0,sizeof(a));
		a.nx = s.w; a.ny = s.h; a.nz = s.d; a.dx = m_dx;
		a.count = (long long) m_particles.size();
		a.particles = m_particles.data();
		a.stride = (int) sizeof(Particle);
		a.offset_position = (int) offsetof(Particle,p);
		a.offset_velocity = (int) offsetof(Particle,velocity);
		a.offset_mass = (int) offsetof(Particle,mass);
		a.offset_apic = m_param.use_apic ? (int) offsetof(Particle,c) : -1;
		a.offset_bullet = (int) offsetof(Particle,bullet);
		a.splat_bullet = m_param.splat_bullet_particle ? 1 : 0;
		for( int dim : DIMS3 ) {
			const size_t nf = s.face(dim).count();
			mass[dim].assign(nf,0.0f); momentum[dim].assign(nf,0.0f); splat_active[dim].assign(nf,0);
			a.mass[dim] = mass[dim].data(); a.momentum[dim] = momentum[dim].data();
			a.splat_active[dim] = splat_active[dim].data();
		}
		const int rc = shkz_b200_splat_host(m_ctx,&a);
		if( rc ) { fail("shkz_b200_splat_host",rc); return; }
		for( int dim : DIMS3 ) {
			const shape3 fs = s.face(dim);
			for( int k=0; k<(int)fs.d; ++k ) for( int j=0; j<(int)fs.h; ++j ) for( int i=0; i<(int)fs.w; ++i ) {
				const size_t n = i+(size_t)fs.w*(j+(size_t)fs.h*k);
				if( splat_active[dim][n] ) mass_and_momentum[dim].set(i,j,k,{mass[dim][n],momentum[dim][n]});
			}
		}
		console::dump( "Done. Took %s\n", timer.stock("splat_momentum").c_str());
	}
	//
	mutable shkz_b200_ctx *m_ctx {nullptr};
	bool m_strict {false};
	int m_device {0};
};
//
extern "C" module * create_instance() {
	return new macnbflip3_b200();
}
//
extern "C" const char *license() {
	return "MIT";
}
