/*
 * macpressuresolver3_b200.cpp -- Shiokaze projection module backed by the
 * B200 CUDA library.
 *
 * Drop-in for Projection=macpressuresolver3: select it with
 * Projection=macpressuresolver3_b200 and the FLIP/APIC liquid and smoke
 * timesteppers call it unchanged. It implements macproject3_interface
 * (include/shiokaze/projection/macproject3_interface.h:42-113) with the
 * meaning of macpressuresolver3 (src/projection/macpressuresolver3.cpp):
 *   - reads the same configuration keys (Residual, MaxIterations,
 *     ModifiedIC, MinDiagRatio, EpsFluid, EpsSolid,
 *     SecondOrderAccurateFluid/Solid) plus B200.* keys;
 *   - project() updates the face velocities in place, switches off the faces
 *     the reference switches off, and keeps the pressure in an array3 that
 *     get_pressure() returns;
 *   - records the same timer labels and the iteration count under
 *     <ArgName>_number_projection_iteration (macpressuresolver3.cpp:253);
 *   - honours the optional terms: surface_tension, set_solid_density,
 *     set_target_volume with Gain (recording <ArgName>_volume_correct_rhs),
 *     and WarmStart, whose previous-solution vector is numbered by the
 *     grids' TileSize exactly as the reference numbers its unknowns and is
 *     serialised through the RCMatrix module's own vector format.
 * The host side only packs the array3/macarray3 grids into dense buffers and
 * calls the C ABI (include/shkz_b200.h); all arithmetic runs on the GPU.
 * Errors never throw: a failed solve is reported on the console and the
 * record, and the velocity is left unprojected with 0 iterations recorded.
 * With B200.Strict=Yes a failure ends the program instead (exit status 1),
 * as the reference's loader does on fatal errors (src/core/module.cpp:141).
 */
#include <shiokaze/array/array3.h>
#include <shiokaze/array/macarray3.h>
#include <shiokaze/projection/macproject3_interface.h>
#include <shiokaze/math/RCMatrix_interface.h>
#include <shiokaze/core/console.h>
#include <shiokaze/core/timer.h>
#include "shkz_b200.h"
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
//
SHKZ_USING_NAMESPACE
//
// Dense staging array in page-locked host memory (shkz_b200_host_alloc), so
// the library's host<->device copies run at full link speed; falls back to
// ordinary heap memory if page-locked memory cannot be had. Grows only.
template <class T> class staging_array {
public:
	staging_array() = default;
	staging_array( const staging_array & ) = delete;
	staging_array &operator=( const staging_array & ) = delete;
	~staging_array() { release(); }
	void assign( size_t n, T value ) {
		resize(n);
		// filled in slices by the host's threads (a 256^3 face grid is 67 MB)
		const size_t nt = std::max(1u,std::min(32u,std::thread::hardware_concurrency()));
		const size_t chunk = (n+nt-1)/nt;
		std::vector<std::thread> workers;
		for( size_t t=0; t<nt; ++t ) {
			const size_t b = t*chunk, e = std::min(n,b+chunk);
			if( b < e ) workers.emplace_back([=]() { std::fill(m_data+b,m_data+e,value); });
		}
		for( auto &w : workers ) w.join();
	}
	void resize( size_t n ) {
		if( n > m_capacity ) {
			release();
			m_data = static_cast<T *>(shkz_b200_host_alloc(n*sizeof(T)));
			m_pinned = m_data != nullptr;
			if( ! m_data ) m_data = new T[n];
			m_capacity = n;
		}
		m_size = n;
	}
	T *data() { return m_data; }
	const T *data() const { return m_data; }
	size_t size() const { return m_size; }
	T &operator[]( size_t i ) { return m_data[i]; }
	const T &operator[]( size_t i ) const { return m_data[i]; }
private:
	void release() {
		if( m_data ) {
			if( m_pinned ) shkz_b200_host_free(m_data);
			else delete [] m_data;
		}
		m_data = nullptr;
		m_capacity = m_size = 0;
	}
	T *m_data {nullptr};
	size_t m_capacity {0}, m_size {0};
	bool m_pinned {false};
};
//
class macpressuresolver3_b200 : public macproject3_interface {
protected:
	//
	LONG_NAME("MAC Pressure Solver 3D (B200)")
	//
	virtual ~macpressuresolver3_b200() {
		if( m_ctx ) shkz_b200_destroy(m_ctx);
	}
	//
	virtual void set_target_volume( double current_volume, double target_volume ) override {
		m_current_volume = current_volume;
		m_target_volume = target_volume;
	}
	//
	virtual void set_solid_density( const macarray3<Real> *solid_density ) override {
		m_solid_density = solid_density;
	}
	//
	// Dense copy of what a(i,j,k) returns for every cell (as array3::linearize
	// builds it: the background value, then the active values, then the fill
	// value of inside cells that are not active) and the active bytes. Only
	// tiles that hold active or filled cells are visited.
	template <class T> static void pack( const array3<T> &a, staging_array<float> &v, staging_array<uint8_t> &m ) {
		const shape3 s = a.shape();
		v.assign(s.count(),(float)a.get_background_value());
		m.assign(s.count(),0);
		a.const_parallel_actives([&]( int i, int j, int k, const typename array3<T>::const_iterator &it ) {
			const size_t n = i+(size_t)s.w*(j+(size_t)s.h*k);
			v[n] = (float)it();
			m[n] = 1;
		});
		a.const_parallel_inside([&]( int i, int j, int k, const typename array3<T>::const_iterator &it ) {
			if( ! it.active()) v[i+(size_t)s.w*(j+(size_t)s.h*k)] = (float)it();
		});
	}
	// A face grid that reads zero everywhere (no active face, zero
	// background, nothing filled) is passed as "no solid velocity".
	static bool reads_zero( const array3<Real> &a ) {
		if( a.get_background_value() != 0.0 || a.count()) return false;
		bool filled (false);
		a.interruptible_const_serial_inside([&](int i, int j, int k, const auto &it) {
			filled = true;
			return true;
		});
		return ! filled;
	}
	//
	virtual void project( double dt,
				macarray3<Real> &velocity,
				const array3<Real> &solid,
				const macarray3<Real> &solid_velocity,
				const array3<Real> &fluid,
				double surface_tension,
				const std::vector<signed_rigidbody3_interface *> *rigidbodies ) override {
		//
		scoped_timer timer(this);
		timer.tick(); console::dump( ">>> Pressure Projection (B200) started...\n" );
		if( ! m_ctx ) {
			int rc = shkz_b200_create(&m_ctx,&m_cfg);
			if( rc ) {
				console::dump( "shkz_b200_create failed: %s\n", shkz_b200_errstr(rc));
				console::write(get_argument_name()+"_number_projection_iteration", 0);
				if( m_strict ) std::exit(1);
				return;
			}
			if( m_prev_pending ) {
				shkz_b200_set_warm_start(m_ctx,m_prev_host.data(),m_prev_host.size());
				m_prev_pending = false;
			}
		} else {
			shkz_b200_set_config(m_ctx,&m_cfg);
		}
		const double vstate[3] = { m_target_volume, m_current_volume, m_y_prev };
		shkz_b200_set_volume_state(m_ctx,vstate);
		//
		timer.tick(); console::dump( "Packing grids..." );
		pack(fluid,m_fluid,m_fluid_active);
		const bool has_solid = levelset_exist_any(solid);
		if( has_solid ) pack(solid,m_solid,m_solid_active);
		bool svel_zero[3];
		for( int dim=0; dim<3; ++dim ) {
			pack(velocity[dim],m_vel[dim],m_vact[dim]);
			svel_zero[dim] = reads_zero(solid_velocity[dim]);
			if( ! svel_zero[dim] ) pack(solid_velocity[dim],m_svel[dim],m_svact[dim]);
			if( m_solid_density ) pack((*m_solid_density)[dim],m_dens[dim],m_dact[dim]);
		}
		console::dump( "Done. Took %s\n", timer.stock("pack_grids").c_str());
		//
		shkz_b200_project_args a;
		std::memset(&a,0,sizeof(a));
		a.nx = m_shape.w; a.ny = m_shape.h; a.nz = m_shape.d;
		a.dx = m_dx; a.dt = dt;
		a.fluid = m_fluid.data(); a.fluid_active = m_fluid_active.data();
		if( has_solid ) { a.solid = m_solid.data(); a.solid_active = m_solid_active.data(); }
		for( int dim=0; dim<3; ++dim ) {
			a.velocity[dim] = m_vel[dim].data();
			a.velocity_active[dim] = m_vact[dim].data();
			a.solid_velocity[dim] = svel_zero[dim] ? nullptr : m_svel[dim].data();
		}
		m_p.resize(m_shape.count());
		m_pact.resize(m_shape.count());
		a.pressure = m_p.data();
		a.pressure_active = m_pact.data();
		a.surface_tension = surface_tension;
		if( m_solid_density ) for( int dim=0; dim<3; ++dim ) a.solid_density[dim] = m_dens[dim].data();
		//
		timer.tick(); console::dump( "Projecting on the GPU...");
		shkz_b200_result res;
		const int rc = shkz_b200_project_host(m_ctx,&a,&res);
		double vnew[3];
		if( shkz_b200_get_volume_state(m_ctx,vnew) == 0 ) m_y_prev = vnew[2];
		if( res.unknowns && m_param.gain && m_target_volume ) {
			console::write(get_argument_name()+"_volume_correct_rhs", res.volume_rhs_correct);
		}
		console::write(get_argument_name()+"_number_projection_iteration", rc ? 0 : res.iterations);
		console::write(get_argument_name()+"_reresid_inf", res.reresid);
		console::write(get_argument_name()+"_reresid_l2", res.reresid_l2);
		if( rc ) {
			console::dump( "failed: %s (%s)\n", shkz_b200_errstr(rc), shkz_b200_last_error(m_ctx));
			if( m_strict ) std::exit(1);
			return;
		}
		// the reference's phase records (macpressuresolver3.cpp:95,168,218,232),
		// from the library's device timings of the same phases
		console::write(get_argument_name()+"_solid_fluid_fractions", res.ms_fractions);
		console::write(get_argument_name()+"_labelling_cells", res.ms_labelling);
		console::write(get_argument_name()+"_build_highres_linsystem", res.ms_build);
		if( res.unknowns && m_param.gain && m_target_volume ) {
			// the correction is added inside the system build's kernel: no time of its own
			console::write(get_argument_name()+"_volume_correction", 0.0);
		}
		console::write(get_argument_name()+"_device_linsolve", res.ms_solve);
		console::write(get_argument_name()+"_device_update_velocity", res.ms_update);
		console::dump( "Done. Took %d iterations, Reresid=%e. Took %s\n", res.iterations, res.reresid, timer.stock("linsolve").c_str());
		//
		timer.tick(); console::dump( "Updating the velocity...");
		// pressure and velocity back into the grids, tile by tile in parallel
		// (parallel_all hands each thread whole tiles, so set() may allocate)
		m_pressure.clear();
		m_pressure.parallel_all([&](int i, int j, int k, auto &it ) {
			const size_t n = i+(size_t)m_shape.w*(j+(size_t)m_shape.h*k);
			if( m_pact[n] ) it.set(m_p[n]);
		});
		velocity.parallel_actives([&](int dim, int i, int j, int k, auto &it, int tn ) {
			const shape3 fs = m_shape.face(dim);
			const size_t n = i+(size_t)fs.w*(j+(size_t)fs.h*k);
			if( m_vact[dim][n] ) it.set(m_vel[dim][n]);
			else it.set_off();
		});
		console::dump( "Done. Took %s\n", timer.stock("update_velocity").c_str());
		console::dump( "<<< Projection done. Took %s.\n", timer.stock("projection").c_str());
	}
	//
	static bool levelset_exist_any( const array3<Real> &levelset ) {
		bool inside (false);
		levelset.interruptible_const_serial_actives([&](int i, int j, int k, const auto &it) {
			if( it() < 0.0 ) inside = true;
			return inside;
		});
		return inside;
	}
	//
	virtual void configure( configuration &config ) override {
		config.get_bool("SecondOrderAccurateFluid",m_param.second_order_accurate_fluid,"Whether to enforce second order accuracy");
		config.get_bool("SecondOrderAccurateSolid",m_param.second_order_accurate_solid,"Whether to enforce second order accuracy for solid surfaces");
		config.get_double("Gain",m_param.gain,"Rate for volume correction");
		config.get_bool("WarmStart",m_param.warm_start,"Start from the solution of previous pressure");
		unsigned tile = m_cfg.index_tile;
		config.get_unsigned("TileSize",tile,"Tile size per dimension");
		m_cfg.index_tile = tile;
		m_cfg.gain = m_param.gain;
		m_cfg.warm_start = m_param.warm_start;
		config.get_double("Residual",m_cfg.residual,"Tolerable residual");
		unsigned max_it = m_cfg.max_iterations;
		config.get_unsigned("MaxIterations",max_it,"Maximal iteration count");
		m_cfg.max_iterations = max_it;
		config.get_double("ModifiedIC",m_cfg.mic_omega,"Modified incomplete cholesky");
		config.get_double("MinDiagRatio",m_cfg.mic_min_diag_ratio,"Minimal diagonal ratio");
		config.get_double("EpsFluid",m_cfg.eps_fluid,"Minimal bound for fluid fraction");
		config.get_double("EpsSolid",m_cfg.eps_solid,"Minimal bound for solid fraction");
		std::string pre ("mic0");
		config.get_string("B200.Preconditioner",pre,"none, mic0 or learned");
		m_cfg.preconditioner = pre == "none" ? SHKZ_B200_PRECOND_NONE : (pre == "learned" ? SHKZ_B200_PRECOND_LEARNED : SHKZ_B200_PRECOND_MIC0);
		bool refine = m_cfg.refine;
		config.get_bool("B200.Refine",refine,"FP64 refinement of the FP32 solve");
		m_cfg.refine = refine;
		int device = m_cfg.device;
		config.get_integer("B200.Device",device,"CUDA device ordinal");
		m_cfg.device = device;
		config.get_bool("B200.Strict",m_strict,"End the program when the GPU projection fails");
		m_cfg.second_order_fluid = m_param.second_order_accurate_fluid;
		m_cfg.second_order_solid = m_param.second_order_accurate_solid;
	}
	virtual void initialize( const shape3 &shape, double dx ) override {
		m_shape = shape;
		m_dx = dx;
	}
	virtual void post_initialize( bool initialized_from_file ) override {
		m_pressure.initialize(m_shape);
		m_target_volume = m_current_volume = m_y_prev = 0.0;
	}
	// Same fields in the same order as macpressuresolver3 (:320-342), the
	// warm-start vector through the RCMatrix module's own vector format, so
	// saved states load in either module.
	virtual void initialize( const filestream &file ) override {
		file.r(m_shape);
		file.r(m_dx);
		file.r(m_target_volume);
		file.r(m_current_volume);
		file.r(m_y_prev);
		if( m_param.warm_start ) {
			auto v = m_factory->allocate_vector();
			v->initialize(file);
			m_prev_host.resize(v->size());
			for( size_t n=0; n<m_prev_host.size(); ++n ) m_prev_host[n] = v->at(n);
			if( m_ctx ) shkz_b200_set_warm_start(m_ctx,m_prev_host.data(),m_prev_host.size());
			else m_prev_pending = true;
		}
	}
	virtual void serialize( const filestream &file ) const override {
		file.w(m_shape);
		file.w(m_dx);
		file.w(m_target_volume);
		file.w(m_current_volume);
		file.w(m_y_prev);
		if( m_param.warm_start ) {
			std::vector<double> prev;
			if( m_ctx ) {
				prev.resize((size_t)std::max(0LL,shkz_b200_warm_start_size(m_ctx)));
				shkz_b200_get_warm_start(m_ctx,prev.data(),prev.size());
			} else {
				prev = m_prev_host;
			}
			auto v = m_factory->allocate_vector(prev.size());
			for( size_t n=0; n<prev.size(); ++n ) v->set(n,prev[n]);
			v->serialize(file);
		}
	}
	virtual const array3<Real> * get_pressure() const override {
		return &m_pressure;
	}
	//
	struct Parameters {
		double gain {1.0};
		bool second_order_accurate_fluid {true};
		bool second_order_accurate_solid {true};
		bool warm_start {false};
	};
	Parameters m_param;
	shkz_b200_config m_cfg = make_default_config();
	static shkz_b200_config make_default_config() {
		shkz_b200_config c;
		shkz_b200_default_config(&c);
		return c;
	}
	shkz_b200_ctx *m_ctx {nullptr};
	bool m_strict {false};
	//
	shape3 m_shape;
	double m_dx {0.0};
	array3<Real> m_pressure{this};
	double m_target_volume {0.0};
	double m_current_volume {0.0};
	double m_y_prev {0.0};
	const macarray3<Real> *m_solid_density {nullptr};
	RCMatrix_factory_driver<size_t,double> m_factory{this,"RCMatrix"};
	std::vector<double> m_prev_host;
	bool m_prev_pending {false};
	// host staging
	staging_array<float> m_fluid, m_solid, m_vel[3], m_svel[3], m_dens[3], m_p;
	staging_array<uint8_t> m_fluid_active, m_solid_active, m_vact[3], m_svact[3], m_dact[3], m_pact;
};
//
extern "C" module * create_instance() {
	return new macpressuresolver3_b200();
}
//
extern "C" const char *license() {
	return "MIT";
}
