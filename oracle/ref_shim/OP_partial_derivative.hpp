/*
 * OP_partial_derivative.hpp -- reconstructed declaration (oracle build only).
 *
 * The reference ships src/common/OP_partial_derivative.cpp but not this header
 * (it is included by rhs_standard.hpp:14 and by the effect_* headers).  The
 * members below are the ones OP_partial_derivative.cpp:4-136 uses, declared in
 * the order its constructor's mem-initialiser list names them (:11-12).
 */
#ifndef OP_PARTIAL_DERIVATIVE_HPP_
#define OP_PARTIAL_DERIVATIVE_HPP_

#include "field.hpp"
#include "grid.hpp"
#include "axis.hpp"
#include "OP_FFT.hpp"
#include "OP_iFFT.hpp"
#include "OP_dealiasing.hpp"

class OP_partial_derivative
{
public :
	OP_partial_derivative(const field_real &field_caller, const direction &e_i);
	OP_partial_derivative(const grid &domain, const direction &e_i);
	OP_partial_derivative(const field_imag &field_caller, const direction &e_i);
	~OP_partial_derivative();
	void operator()(const field_imag &in, field_imag &out);
private :
	OP_FFT my_FFT;
	OP_iFFT my_iFFT;
	field_real Buffer;
	OP_dealiasing my_dealiasing;
	axis * my_axis;
	int * my_X;
	int my_i;
	int my_j;
	int my_k;
	bool IsLinear;
	double * k_val;
	double * dS_val;
};

#endif
