// Harness-side linear-solver module for the compiled reference (test
// infrastructure only; never part of the product).
//
// Selected with LinSolver=refmic0. It reads the assembled RCMatrix exactly as
// the reference's src/linsolver/pcg.cpp:47-55 does, optionally dumps A (CSR)
// and b, and then solves in one of two modes:
//   RefMode=shipped : the reference's PCGSolver<double> unchanged
//                     (local/include/pcgsolver/pcg_solver.h:246-295); its
//                     preconditioner result is discarded (:379-384), so this
//                     is plain CG.
//   RefMode=mic0    : the same loop with the header's own MIC(0) factor and
//                     triangular sweeps applied (pcg_solver.h:88-223). This is
//                     the preconditioner the reference intends to ship.
// The stopping rule is the reference's ||r||_inf <= tol*||b||_inf with x0=0.
#include <shiokaze/linsolver/RCMatrix_solver.h>
#include <pcgsolver/pcg_solver.h>
#include <cstdio>
#include <cstdlib>
#include <chrono>
//
SHKZ_USING_NAMESPACE
//
namespace {
// PCG loop of pcg_solver.h:246-295 with the MIC(0) preconditioner kept.
template <class T>
bool mic0_pcg( const SparseMatrix<T> &matrix, const std::vector<T> &rhs, std::vector<T> &result,
			   T tolerance_factor, int max_iterations, T omega, T min_ratio,
			   T &residual_out, int &iterations_out ) {
	unsigned n = matrix.n;
	std::vector<T> z(n), s(n), r(n);
	SparseColumnLowerFactor<T> ic;
	FixedSparseMatrix<T> fixed;
	result.assign(n,0);
	r = rhs;
	residual_out = BLAS::abs_max(r);
	T residual0 = residual_out;
	if( residual_out == 0 ) { iterations_out = 0; return true; }
	double tol = tolerance_factor*residual_out;
	factor_modified_incomplete_cholesky0(matrix,ic,omega,min_ratio);
	auto apply = [&]( const std::vector<T> &x, std::vector<T> &out ) {
		solve_lower(ic,x,out);
		solve_lower_transpose_in_place(ic,out);
	};
	apply(r,z);
	double rho = BLAS::dot(z,r);
	if( rho == 0 || rho != rho ) { iterations_out = 0; return false; }
	s = z;
	fixed.construct_from_matrix(matrix);
	int it;
	for( it=0; it<max_iterations; ++it ) {
		multiply(fixed,s,z);
		double alpha = rho/BLAS::dot(s,z);
		BLAS::add_scaled(alpha,s,result);
		BLAS::add_scaled(-alpha,z,r);
		residual_out = BLAS::abs_max(r);
		if( residual_out <= tol ) {
			iterations_out = it+1;
			residual_out /= residual0;
			return true;
		}
		apply(r,z);
		double rho_new = BLAS::dot(z,r);
		double beta = rho_new/rho;
		BLAS::add_scaled(beta,s,z); s.swap(z);
		rho = rho_new;
	}
	iterations_out = it;
	residual_out /= residual0;
	return false;
}
}
//
template <class N, class T> class refmic0_solver : public RCMatrix_solver_interface<N,T> {
protected:
	LONG_NAME("Reference MIC(0) PCG harness")
	ARGUMENT_NAME("PCG")
	//
	virtual void configure( configuration &config ) override {
		config.get_double("Residual",m_residual,"Tolerable residual");
		config.get_unsigned("MaxIterations",m_max_iterations,"Maximal iteration count");
		config.get_string("RefMode",m_mode,"shipped or mic0");
	}
	virtual typename RCMatrix_solver_interface<N,T>::Result solve( const RCMatrix_interface<N,T> *A, const RCMatrix_vector_interface<N,T> *b, RCMatrix_vector_interface<N,T> *x ) const override {
		//
		SparseMatrix<T> matrix(A->rows());
		for( N row=0; row<matrix.n; ++row ) {
			A->const_for_each(row,[&]( N column, T value ) {
				matrix.add_to_element(row,column,value);
			});
		}
		std::vector<T> rhs;
		b->convert_to(rhs);
		//
		const char *dump = std::getenv("SHKZ_REF_DUMP");
		if( dump && *dump ) {
			std::string path = std::string(dump)+".system.bin";
			FILE *fp = std::fopen(path.c_str(),"wb");
			if( fp ) {
				unsigned long long n = matrix.n, nnz = 0;
				for( unsigned i=0; i<matrix.n; ++i ) nnz += matrix.index[i].size();
				std::fwrite(&n,8,1,fp); std::fwrite(&nnz,8,1,fp);
				unsigned long long acc = 0;
				for( unsigned i=0; i<matrix.n; ++i ) { std::fwrite(&acc,8,1,fp); acc += matrix.index[i].size(); }
				std::fwrite(&acc,8,1,fp);
				for( unsigned i=0; i<matrix.n; ++i ) for( auto c : matrix.index[i] ) { unsigned long long cc=c; std::fwrite(&cc,8,1,fp); }
				for( unsigned i=0; i<matrix.n; ++i ) std::fwrite(matrix.value[i].data(),sizeof(T),matrix.value[i].size(),fp);
				std::fwrite(rhs.data(),sizeof(T),rhs.size(),fp);
				std::fclose(fp);
			}
		}
		//
		std::vector<T> result(matrix.n);
		T residual_out (0);
		int iterations_out (0);
		auto t0 = std::chrono::steady_clock::now();
		if( m_mode == "shipped" ) {
			PCGSolver<T> solver;
			solver.set_solver_parameters(m_residual,m_max_iterations);
			solver.solve(matrix,rhs,result,residual_out,iterations_out);
		} else {
			mic0_pcg<T>(matrix,rhs,result,m_residual,m_max_iterations,0.97,0.25,residual_out,iterations_out);
		}
		auto t1 = std::chrono::steady_clock::now();
		m_last_solve_ms = std::chrono::duration<double,std::milli>(t1-t0).count();
		x->convert_from(result);
		if( dump && *dump ) {
			std::string path = std::string(dump)+".solve.txt";
			FILE *fp = std::fopen(path.c_str(),"w");
			if( fp ) {
				std::fprintf(fp,"%d %.17g %.6f\n",iterations_out,(double)residual_out,m_last_solve_ms);
				std::fclose(fp);
			}
		}
		return {(N)iterations_out,(T)residual_out};
	}
	double m_residual {1e-4};
	unsigned m_max_iterations {30000};
	std::string m_mode {"mic0"};
	mutable double m_last_solve_ms {0.0};
};
//
extern "C" module * create_instance() {
	return new refmic0_solver<size_t,double>();
}
extern "C" const char *license() {
	return "test harness";
}
