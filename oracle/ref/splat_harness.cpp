// Driver that runs the compiled reference FLIP splat (test infrastructure
// only). It fills the reference's own macnbflip3 (src/flip/macnbflip3.cpp,
// compiled into this binary from where it lies) with particles from an input
// file, lets it hash them (sort_particles, :746-757, through the
// pointgridhash3 module) and calls
//   splat(time, mass_and_momentum)                   (:103-148)
// then combines the splatted momentum with the grid velocity as the liquid
// solver does right before its projection (src/liquid/macflipliquid3.cpp:
// 135-151: grid mass = max(0, 1 - particle mass) where the grid face is
// active, else 0; u = (grid mass * u + momentum) / (grid mass + mass) on
// every face the splat left active, which then becomes active).
//
// usage: shkz_ref_splat <in.bin> <out.bin> [Key=Value ...]
//   prints "hash_ms H splat_ms S combine_ms C": wall time of the particle
//   hash (sort_particles), the splat and the combined velocity
//   configuration keys go to the reference (APIC=Yes|No,
//   SplatBulletParticle=Yes|No, ...). With FLIP=<module> the splat is that
//   FLIP module's, loaded by the reference's module loader (e.g. the B200
//   module macnbflip3_b200): the particles reach it through the reference's
//   own serialisation (recursive_serialize of the compiled-in macnbflip3, then
//   recursive_initialize of the module from that file), and the splat runs
//   through macflip3_interface::splat.
//
// Input file (little endian):
//   char[8] "SHKZSP01"; int32 nx, ny, nz; double dx, time; int64 count;
//   float p[count*3], c[count*9] (c[dim][component]), velocity[count*3],
//   mass[count]; uint8 bullet[count];
//   for dim in 0..2: float u[face count]; uint8 u_set[face count]
// Output file:
//   for dim in 0..2: float mass[fc], momentum[fc]; uint8 splat_active[fc];
//                    float u[fc] (effective value); uint8 u_active[fc]
// Faces are x-fastest (i + W*(j + H*k)) on the dim's face grid.
#include "macnbflip3.h"
#include <shiokaze/array/macarray3.h>
#include <shiokaze/core/configuration.h>
#include <shiokaze/core/credit.h>
#include <shiokaze/core/filesystem.h>
#include <chrono>
#include <cstdio>
#include <cstring>
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
// the reference's particle storage is protected; a subclass fills it
class flip_access : public macnbflip3 {
public:
	using macnbflip3::Particle;
	void run_splat( double time, macarray3<macflip3_interface::mass_momentum3> &mm ) const { splat(time,mm); }
	void load_particles( const std::vector<Particle> &particles ) {
		m_particles = particles;
		sort_particles();
	}
	static Particle blank() { return Particle(); }
};
//
// the FLIP module named by the FLIP key, through the reference's loader
class module_root : public recursive_configurable {
public:
	macflip3_driver m_flip{this,"macnbflip3"};
};
//
class splat_root : public recursive_configurable {
public:
	splat_root() {
		add_child(&m_flip);
		set_environment("shape",&m_shape);
		set_environment("dx",&m_dx);
	}
	shape3 m_shape;
	double m_dx {1.0};
	flip_access m_flip;
	macarray3<Real> m_velocity{this};
	macarray3<macflip3_interface::mass_momentum3> m_mass_momentum{this};
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
	int hdr[3];
	double dhdr[2];
	long long count;
	if( ! rd(fp,magic,8) || std::memcmp(magic,"SHKZSP01",8) || ! rd(fp,hdr,3) || ! rd(fp,dhdr,2) || ! rd(fp,&count,1) ) {
		std::fprintf(stderr,"bad header\n"); return 2;
	}
	const int nx=hdr[0], ny=hdr[1], nz=hdr[2];
	const double dx=dhdr[0], time=dhdr[1];
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
	splat_root root;
	root.m_shape = shape;
	root.m_dx = dx;
	root.recursive_load(config);
	root.recursive_configure(config);
	root.recursive_initialize();
	//
	std::vector<float> p(count*3), c(count*9), v(count*3), m(count);
	std::vector<unsigned char> bullet(count);
	if( ! rd(fp,p.data(),p.size()) || ! rd(fp,c.data(),c.size()) || ! rd(fp,v.data(),v.size()) ||
		! rd(fp,m.data(),m.size()) || ! rd(fp,bullet.data(),bullet.size())) {
		std::fprintf(stderr,"short particles\n"); return 2;
	}
	std::vector<flip_access::Particle> particles(count,flip_access::blank());
	for( long long n=0; n<count; ++n ) {
		auto &q = particles[n];
		for( int a=0; a<3; ++a ) {
			q.p[a] = p[3*n+a];
			q.velocity[a] = v[3*n+a];
			for( int b=0; b<3; ++b ) q.c[a][b] = c[9*n+3*a+b];
		}
		q.mass = m[n];
		q.r = 0.25*dx;
		q.bullet = bullet[n];
	}
	const auto t0 = std::chrono::steady_clock::now();
	root.m_flip.load_particles(particles);
	const auto t1 = std::chrono::steady_clock::now();
	//
	auto &velocity = root.m_velocity;
	velocity.initialize(shape);
	for( int dim : DIMS3 ) {
		const shape3 fs = shape.face(dim);
		const size_t nf = fs.count();
		std::vector<float> u(nf);
		std::vector<unsigned char> set(nf);
		if( ! rd(fp,u.data(),nf) || ! rd(fp,set.data(),nf)) { std::fprintf(stderr,"short velocity\n"); return 2; }
		for( int k=0; k<(int)fs.d; ++k ) for( int j=0; j<(int)fs.h; ++j ) for( int i=0; i<(int)fs.w; ++i ) {
			size_t n = i+(size_t)fs.w*(j+(size_t)fs.h*k);
			if( set[n] ) velocity[dim].set(i,j,k,u[n]);
		}
	}
	std::fclose(fp);
	//
	auto &mm = root.m_mass_momentum;
	mm.initialize(shape);
	module_root froot;
	const bool use_module = dict.count("FLIP") > 0;
	if( use_module ) {
		const std::string path = std::string(argv[2])+".flip";
		{
			filestream out(path,filestream::WRITE);
			root.m_flip.recursive_serialize(out);
		}
		froot.recursive_load(config);
		froot.recursive_configure(config);
		filestream in(path,filestream::READ);
		froot.m_flip->recursive_initialize(in);
	}
	const auto t2 = std::chrono::steady_clock::now();
	if( use_module ) froot.m_flip->splat(time,mm);
	else root.m_flip.run_splat(time,mm);
	const auto t3 = std::chrono::steady_clock::now();
	//
	// combined grid velocity: every value is computed from the velocity
	// before any is written, then all are written
	std::vector<std::vector<Real> > combined(3);
	for( int dim : DIMS3 ) {
		const shape3 fs = shape.face(dim);
		combined[dim].assign(fs.count(),0.0f);
		mm[dim].const_serial_actives([&]( int i, int j, int k, const auto &it ) {
			const auto value = it();
			const Real grid_mass = velocity[dim].active(i,j,k) ? std::max(0.0,1.0-value.mass) : 0.0;
			combined[dim][i+(size_t)fs.w*(j+(size_t)fs.h*k)] =
				(grid_mass*velocity[dim](i,j,k)+value.momentum)/(grid_mass+value.mass);
		});
	}
	for( int dim : DIMS3 ) {
		const shape3 fs = shape.face(dim);
		mm[dim].const_serial_actives([&]( int i, int j, int k, const auto &it ) {
			velocity[dim].set(i,j,k,combined[dim][i+(size_t)fs.w*(j+(size_t)fs.h*k)]);
		});
	}
	const auto t4 = std::chrono::steady_clock::now();
	auto ms = []( auto a, auto b ) { return std::chrono::duration<double,std::milli>(b-a).count(); };
	std::printf("hash_ms %.6f splat_ms %.6f combine_ms %.6f\n",ms(t0,t1),ms(t2,t3),ms(t3,t4));
	//
	FILE *out = std::fopen(argv[2],"wb");
	if( ! out ) { std::fprintf(stderr,"cannot write %s\n",argv[2]); return 2; }
	for( int dim : DIMS3 ) {
		const shape3 fs = shape.face(dim);
		const size_t nf = fs.count();
		std::vector<float> mass(nf), mom(nf), u(nf);
		std::vector<unsigned char> sa(nf), ua(nf);
		for( int k=0; k<(int)fs.d; ++k ) for( int j=0; j<(int)fs.h; ++j ) for( int i=0; i<(int)fs.w; ++i ) {
			size_t n = i+(size_t)fs.w*(j+(size_t)fs.h*k);
			sa[n] = mm[dim].active(i,j,k);
			if( sa[n] ) {
				const auto value = mm[dim](i,j,k);
				mass[n] = value.mass;
				mom[n] = value.momentum;
			}
			u[n] = velocity[dim](i,j,k);
			ua[n] = velocity[dim].active(i,j,k);
		}
		wr(out,mass.data(),nf); wr(out,mom.data(),nf); wr(out,sa.data(),nf);
		wr(out,u.data(),nf); wr(out,ua.data(),nf);
	}
	std::fclose(out);
	return 0;
}
