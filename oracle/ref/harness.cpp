// Driver that runs the compiled reference projection (test infrastructure
// only). It builds the reference's own array3/macarray3 grids from a dense
// input file, loads Projection=macpressuresolver3 through the reference's
// module loader (src/core/module.cpp:103-172) and calls
//   project(dt, velocity, solid, solid_velocity, fluid)
// (src/projection/macpressuresolver3.cpp:54-299). It then writes what the
// reference grids hold after the call: effective values and active bits of
// the inputs, pressure and its active bits, and the projected face velocities
// and their active bits.
//
// usage: shkz_ref_harness <in.bin> <out.bin> [Key=Value ...]
//
// Harness keys (the rest go to the reference's configuration):
//   HarnessRepeat=N            project N times (velocity reset between them;
//                              WarmStart=Yes carries the previous solution)
//   HarnessSurfaceTension=k    surface_tension argument of project()
//   HarnessDensity=<file>      set_solid_density() with face densities read
//                              from <file> (double, x-fastest, dim 0..2)
//   HarnessVolume=<cur>:<tgt>  set_target_volume(cur, tgt) before each call
//   HarnessExtend=w            after the last projection, extend the velocity
//                              w layers with macarray_extrapolator3::extrapolate
//                              (include/shiokaze/array/macarray_extrapolator3.h)
//   HarnessConstrain=1         then macutility3::constrain_velocity(solid, velocity)
//   HarnessProject=0           no projection (the extension then runs on the
//                              input velocity; the pressure is written empty)
//   Projection=<module>        any projection module (default macpressuresolver3;
//                              macstreamfuncsolver3 has no pressure grid, which is
//                              then written as empty)
//                              (src/utility/macutility3.cpp:61-92), as
//                              macliquid3::extend_both does (src/liquid/macliquid3.cpp:330-340)
//
// Input file (little endian):
//   char[8] "SHKZIN01"; int32 nx,ny,nz, has_solid, has_solid_velocity;
//   double dx, dt, fluid_band, solid_band;
//   double fluid[nx*ny*nz];          uint8 fluid_set[nx*ny*nz]
//   if has_solid: double solid[(nx+1)(ny+1)(nz+1)]; uint8 solid_set[...]
//   for dim in 0..2: double u_dim[face count]; uint8 u_set[face count]
//   if has_solid_velocity: for dim: double us_dim[face count]
// Grids are x-fastest (i + nx*(j + ny*k)). A cell is set (made active) only
// where *_set is 1. Level sets are then marked with set_as_levelset(band)
// and flood filled, as macutility3::assign_initial_variables does
// (src/utility/macutility3.cpp:354-375, 399-416).
#include <shiokaze/array/array3.h>
#include <shiokaze/array/macarray3.h>
#include <shiokaze/projection/macproject3_interface.h>
#include <shiokaze/utility/macutility3_interface.h>
#include <shiokaze/array/macarray_extrapolator3.h>
#include <shiokaze/core/configuration.h>
#include <shiokaze/core/credit.h>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <chrono>
#include <map>
#include <string>
#include <vector>
//
SHKZ_USING_NAMESPACE
//
namespace {
template <class T> bool rd( FILE *fp, T *p, size_t n ) { return std::fread(p,sizeof(T),n,fp) == n; }
template <class T> void wr( FILE *fp, const T *p, size_t n ) { std::fwrite(p,sizeof(T),n,fp); }
//
class harness_root : public recursive_configurable {
public:
	harness_root() {
		m_macproject.set_environment("shape",&m_shape);
		m_macproject.set_environment("dx",&m_dx);
		m_macutility.set_environment("shape",&m_shape);
		m_macutility.set_environment("dx",&m_dx);
	}
	shape3 m_shape;
	double m_dx {1.0};
	array3<Real> m_fluid{this};
	array3<Real> m_solid{this};
	macarray3<Real> m_velocity{this};
	macarray3<Real> m_solid_velocity{this};
	macarray3<Real> m_density{this};
	array3<Real> m_no_pressure{this};
	macproject3_driver m_macproject{this,"macpressuresolver3"};
	macutility3_driver m_macutility{this,"macutility3"};
};
}
//
int main( int argc, const char *argv[] ) {
	//
	if( argc < 3 ) {
		std::fprintf(stderr,"usage: %s in.bin out.bin [Key=Value ...]\n",argv[0]);
		return 2;
	}
	FILE *fp = std::fopen(argv[1],"rb");
	if( ! fp ) { std::fprintf(stderr,"cannot open %s\n",argv[1]); return 2; }
	char magic[8];
	int hdr[5];
	double dhdr[4];
	if( ! rd(fp,magic,8) || std::memcmp(magic,"SHKZIN01",8) || ! rd(fp,hdr,5) || ! rd(fp,dhdr,4) ) {
		std::fprintf(stderr,"bad header\n"); return 2;
	}
	const int nx=hdr[0], ny=hdr[1], nz=hdr[2];
	const bool has_solid = hdr[3], has_solid_velocity = hdr[4];
	const double dx=dhdr[0], dt=dhdr[1], fluid_band=dhdr[2], solid_band=dhdr[3];
	const shape3 shape(nx,ny,nz);
	//
	std::map<std::string,std::string> dict;
	for( int n=3; n<argc; ++n ) {
		std::string s(argv[n]);
		auto pos = s.find('=');
		if( pos != std::string::npos ) dict[s.substr(0,pos)] = s.substr(pos+1);
	}
	configuration config(dict);
	credit root_credit("Root","Root");
	configuration::auto_group group(config,root_credit);
	harness_root root;
	root.m_shape = shape;
	root.m_dx = dx;
	root.recursive_load(config);
	root.recursive_configure(config);
	root.recursive_initialize();
	//
	auto &fluid = root.m_fluid;
	auto &solid = root.m_solid;
	auto &velocity = root.m_velocity;
	auto &solid_velocity = root.m_solid_velocity;
	//
	const size_t nc = shape.count();
	std::vector<double> buf;
	std::vector<unsigned char> mask;
	//
	fluid.initialize(shape);
	buf.resize(nc); mask.resize(nc);
	if( ! rd(fp,buf.data(),nc) || ! rd(fp,mask.data(),nc)) { std::fprintf(stderr,"short fluid\n"); return 2; }
	for( int k=0; k<nz; ++k ) for( int j=0; j<ny; ++j ) for( int i=0; i<nx; ++i ) {
		size_t n = i+(size_t)nx*(j+(size_t)ny*k);
		if( mask[n] ) fluid.set(i,j,k,buf[n]);
	}
	fluid.set_as_levelset(fluid_band);
	fluid.flood_fill();
	//
	const shape3 nshape = shape.nodal();
	solid.initialize(nshape,1.0);
	if( has_solid ) {
		const size_t nn = nshape.count();
		buf.resize(nn); mask.resize(nn);
		if( ! rd(fp,buf.data(),nn) || ! rd(fp,mask.data(),nn)) { std::fprintf(stderr,"short solid\n"); return 2; }
		for( int k=0; k<nz+1; ++k ) for( int j=0; j<ny+1; ++j ) for( int i=0; i<nx+1; ++i ) {
			size_t n = i+(size_t)(nx+1)*(j+(size_t)(ny+1)*k);
			if( mask[n] ) solid.set(i,j,k,buf[n]);
		}
		solid.set_as_levelset(solid_band);
		solid.flood_fill();
	}
	//
	velocity.initialize(shape);
	solid_velocity.initialize(shape);
	std::vector<double> vel_in[3];
	std::vector<unsigned char> vel_mask[3];
	for( int dim=0; dim<3; ++dim ) {
		const size_t nf = shape.face(dim).count();
		vel_in[dim].resize(nf); vel_mask[dim].resize(nf);
		if( ! rd(fp,vel_in[dim].data(),nf) || ! rd(fp,vel_mask[dim].data(),nf)) { std::fprintf(stderr,"short velocity\n"); return 2; }
	}
	auto set_velocity = [&]() {
		velocity.clear();
		for( int dim=0; dim<3; ++dim ) {
			const shape3 fs = shape.face(dim);
			for( int k=0; k<fs.d; ++k ) for( int j=0; j<fs.h; ++j ) for( int i=0; i<fs.w; ++i ) {
				size_t n = i+(size_t)fs.w*(j+(size_t)fs.h*k);
				if( vel_mask[dim][n] ) velocity[dim].set(i,j,k,vel_in[dim][n]);
			}
		}
	};
	set_velocity();
	if( has_solid_velocity ) {
		for( int dim=0; dim<3; ++dim ) {
			const shape3 fs = shape.face(dim);
			const size_t nf = fs.count();
			buf.resize(nf);
			if( ! rd(fp,buf.data(),nf)) { std::fprintf(stderr,"short solid velocity\n"); return 2; }
			for( int k=0; k<fs.d; ++k ) for( int j=0; j<fs.h; ++j ) for( int i=0; i<fs.w; ++i ) {
				size_t n = i+(size_t)fs.w*(j+(size_t)fs.h*k);
				if( buf[n] != 0.0 ) solid_velocity[dim].set(i,j,k,buf[n]);
			}
		}
	}
	std::fclose(fp);
	//
	const double kappa = dict.count("HarnessSurfaceTension") ? std::atof(dict["HarnessSurfaceTension"].c_str()) : 0.0;
	if( dict.count("HarnessDensity") ) {
		FILE *df = std::fopen(dict["HarnessDensity"].c_str(),"rb");
		if( ! df ) { std::fprintf(stderr,"cannot open density file\n"); return 2; }
		root.m_density.initialize(shape);
		for( int dim=0; dim<3; ++dim ) {
			const shape3 fs = shape.face(dim);
			buf.resize(fs.count());
			if( ! rd(df,buf.data(),buf.size())) { std::fprintf(stderr,"short density\n"); return 2; }
			for( int k=0; k<fs.d; ++k ) for( int j=0; j<fs.h; ++j ) for( int i=0; i<fs.w; ++i ) {
				root.m_density[dim].set(i,j,k,buf[i+(size_t)fs.w*(j+(size_t)fs.h*k)]);
			}
		}
		std::fclose(df);
		root.m_macproject->set_solid_density(&root.m_density);
	}
	double vol_cur (0.0), vol_tgt (0.0);
	const bool has_volume = dict.count("HarnessVolume") > 0;
	if( has_volume ) std::sscanf(dict["HarnessVolume"].c_str(),"%lf:%lf",&vol_cur,&vol_tgt);
	//
	FILE *out = std::fopen(argv[2],"wb");
	if( ! out ) { std::fprintf(stderr,"cannot open %s\n",argv[2]); return 2; }
	wr(out,"SHKZOUT1",8);
	int ohdr[4] = {nx,ny,nz,(int)sizeof(Real)};
	wr(out,ohdr,4);
	// effective inputs as the reference reads them
	auto dump_cells = [&]( const array3<Real> &a, const shape3 &s ) {
		std::vector<double> v(s.count());
		std::vector<unsigned char> m(s.count());
		for( int k=0; k<s.d; ++k ) for( int j=0; j<s.h; ++j ) for( int i=0; i<s.w; ++i ) {
			size_t n = i+(size_t)s.w*(j+(size_t)s.h*k);
			v[n] = a(i,j,k);
			m[n] = a.active(i,j,k);
		}
		wr(out,v.data(),v.size());
		wr(out,m.data(),m.size());
	};
	dump_cells(fluid,shape);
	dump_cells(solid,nshape);
	for( int dim=0; dim<3; ++dim ) dump_cells(velocity[dim],shape.face(dim));
	//
	const int repeat = dict.count("HarnessRepeat") ? std::atoi(dict["HarnessRepeat"].c_str()) : 1;
	const bool project = ! dict.count("HarnessProject") || std::atoi(dict["HarnessProject"].c_str());
	double best_ms = project ? 1e300 : 0.0;
	for( int rep=0; project && rep<std::max(1,repeat); ++rep ) {
		if( rep ) set_velocity();
		if( has_volume ) root.m_macproject->set_target_volume(vol_cur,vol_tgt);
		auto t0 = std::chrono::steady_clock::now();
		root.m_macproject->project(dt,velocity,solid,solid_velocity,fluid,kappa);
		auto t1 = std::chrono::steady_clock::now();
		best_ms = std::min(best_ms,std::chrono::duration<double,std::milli>(t1-t0).count());
	}
	//
	if( dict.count("HarnessExtend") ) {
		const int width = std::atoi(dict["HarnessExtend"].c_str());
		if( width > 0 ) macarray_extrapolator3::extrapolate<Real>(velocity,width);
		if( dict.count("HarnessConstrain") && std::atoi(dict["HarnessConstrain"].c_str()) ) {
			root.m_macutility->constrain_velocity(solid,velocity);
		}
	}
	//
	// a projection without a pressure grid (macstreamfuncsolver3::get_pressure
	// returns nullptr) is written as an empty, inactive grid
	const array3<Real> *pressure_ptr = project ? root.m_macproject->get_pressure() : nullptr;
	if( ! pressure_ptr ) {
		root.m_no_pressure.initialize(shape);
		pressure_ptr = &root.m_no_pressure;
	}
	dump_cells(*pressure_ptr,shape);
	for( int dim=0; dim<3; ++dim ) dump_cells(velocity[dim],shape.face(dim));
	wr(out,&best_ms,1);
	std::fclose(out);
	std::printf("projection_ms %.3f\n",best_ms);
	return 0;
}
