// project_probe - test harness linked against the reference library built
// from source (oracle/_ref): Bimage::project (bsoft/src/img/Bimage_project.cpp:
// 362-443) of a map for a list of views with the FSI kernel, back-transformed
// to real space (conversion 1, real part), as bproject -kernel does.
// Usage: project_probe map.mrc resolution views.txt out.raw [width power]
// views.txt: "x y z angle(rad)" per view; out.raw: float32 n x N x N.
#include "rwimg.h"
#include "Bimage.h"
#include "FSI_Kernel.h"
#include "View.h"
#include "utilities.h"
#include "linked_list.h"
#include <fstream>

extern int verbose;

int main(int argc, char** argv) {
	if ( argc < 5 ) { std::cerr << "usage: project_probe map res views out [w p]" << std::endl; return 1; }
	verbose = 0;
	Bimage* p = read_img(argv[1], 1, -1);
	if ( !p ) return 2;
	double res = atof(argv[2]);
	int kw = argc > 5 ? atoi(argv[5]) : 8, kp = argc > 6 ? atoi(argv[6]) : 2;
	View* views = NULL;
	View* last = NULL;
	{ std::ifstream f(argv[3]); double x, y, z, a;
	  while ( f >> x >> y >> z >> a ) {
		View* v = (View *) add_item((char **) &views, sizeof(View));
		*v = View(x, y, z, a);
		last = v;
	  } }
	(void)last;
	FSI_Kernel* kernel = new FSI_Kernel(kw, kp);
	Bimage* proj = p->project(views, res, kernel, 0, 1, Real);
	std::ofstream o(argv[4], std::ios::binary);
	o.write((const char*)proj->data_pointer(), sizeof(float)*proj->image_size()*proj->images());
	std::cout << "n " << proj->images() << " size " << proj->sizeX() << " " << proj->sizeY()
		<< " origin " << proj->image->origin()[0] << " " << proj->image->origin()[1] << std::endl;
	return 0;
}
