// Reference harness: drives the reference TAPSim classes (built from the
// reference's own sources by oracle/Makefile) to produce golden data for the
// test suite and the CPU leg of bench.py.  This file is test infrastructure:
// nothing in the product links it.
//
// The event loop below restates the order of steps I-VI of
// Process::evaporation (tapsim/process.cpp:680-1036) using the reference's own
// functions, and adds what the checker needs: the top-two evaporation
// probabilities of every event (near-tie margin), an optional forced removal
// sequence (so that a device run that diverges at a near-tie can be compared
// event by event), per-event wall time and potential snapshots.
//
// Commands
//   ref_harness mesh <cfg> <nodes> <dump_out>
//       Process::initialization (readConfig, readGeomGrid, tetrahedralize,
//       fastSync) then File_Io::writeSystem.
//   ref_harness evap <cfg> <nodes|-> <ini> <n_events> <events_out> [options]
//       --dump <file>        resume from a TAPSIM dump instead of a node file
//       --threads <n>        relaxation threads (reference --threads)
//       --init-relax thr cycle queue   initial relaxation (default: refresh
//                            parameters of the ini, as EvaporationCommands
//                            ::setDefaults does, commands.cpp:931-933)
//       --no-init-relax
//       --force <file>       node indices to remove, one per line
//       --phi <file>         write float32 potential() of all nodes after the
//                            initial relaxation
//       --phi-events <file>  append float32 potentials after every event
//       --no-sync            with --dump: keep the dump's couplings (resumption)
//       --trajectories <file> <ascii|binary> <chunk>
//                            write every event's trajectory with the
//                            reference's own File_Io::LogTrajectory, as
//                            process.cpp:1048-1049 pushes it
//       --grids <file> <ascii|binary>
//       --surfaces <file> <ascii|binary> <neighbours 0|1>
//                            snapshots after every event with the reference's
//                            own File_Io::LogGrid / LogSurface
//                            (process.cpp:1068-1072 with interval 1)

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <queue>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>
#include <sys/time.h>

#include "system_3d.h"
#include "surface_3d.h"
#include "trajectory_3d.h"
#include "process.h"
#include "file_io.h"
#include "logTrajectory.h"
#include "logGrid.h"
#include "logSurface.h"

// commands.cpp (linked for makeIniList) refers to these globals, which the
// reference defines next to main() in tapsim.cpp.
const char* tapSimVersion = "1.0b";
const char* tapSimRevision = "3225";
const char* tapSim_distVersion = "ref_harness";
const char* tapSim_distDate = __DATE__;
const char* tapSim_distTime = __TIME__;
const char* uniqueDate = __DATE__;
const char* uniqueTime = __TIME__;
const char* defaultIniFilename = "tapsim.ini";

static double wall_seconds()
{
	struct timeval tv;
	gettimeofday(&tv, 0);
	return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static void write_phi(FILE* f, const System_3d& system)
{
	const int n = system.gridTable.numNodes();
	std::vector<float> phi(n);
	for (int i = 0; i < n; i++) phi[i] = system.gridTable.potential(i);
	fwrite(&phi[0], sizeof(float), n, f);
}

static int cmd_mesh(int argc, char** argv)
{
	if (argc < 5) { fprintf(stderr, "usage: ref_harness mesh cfg nodes dump\n"); return 2; }
	System_3d system;
	system.gridTable.setThreadNum(1);
	Process::initialization(argv[2], argv[3], &system);
	File_Io::writeSystem(argv[4], system, 0);
	printf("nodes %d tets %d\n", system.geomTable.numNodes(), system.geomTable.numTetrahedra());
	return 0;
}

static int cmd_evap(int argc, char** argv)
{
	if (argc < 7) { fprintf(stderr, "usage: ref_harness evap cfg nodes ini n_events out [options]\n"); return 2; }
	const char* cfg = argv[2];
	const char* nodes = argv[3];
	const char* ini = argv[4];
	const int nEvents = atoi(argv[5]);
	const char* outName = argv[6];

	const char* dumpIn = 0;
	const char* forceName = 0;
	const char* phiName = 0;
	const char* phiEventsName = 0;
	int threads = 1;
	const char* trajName = 0;
	int trajMode = File_Io::ASCII;
	unsigned trajChunk = 0;
	const char* gridName = 0;
	int gridMode = File_Io::ASCII;
	const char* surfName = 0;
	int surfMode = File_Io::ASCII;
	bool surfNeighbours = false;
	int initRelax = 1;
	bool initGiven = false;
	bool noSync = false;
	float initThr = 0.0f;
	unsigned initCycle = 0, initQueue = 0;

	for (int a = 7; a < argc; a++)
	{
		if (!strcmp(argv[a], "--dump")) dumpIn = argv[++a];
		else if (!strcmp(argv[a], "--threads")) threads = atoi(argv[++a]);
		else if (!strcmp(argv[a], "--no-init-relax")) initRelax = 0;
		else if (!strcmp(argv[a], "--init-relax"))
		{
			initGiven = true;
			initThr = atof(argv[++a]);
			initCycle = atoi(argv[++a]);
			initQueue = atoi(argv[++a]);
		}
		else if (!strcmp(argv[a], "--force")) forceName = argv[++a];
		else if (!strcmp(argv[a], "--phi")) phiName = argv[++a];
		else if (!strcmp(argv[a], "--phi-events")) phiEventsName = argv[++a];
		else if (!strcmp(argv[a], "--no-sync")) noSync = true;
		else if (!strcmp(argv[a], "--trajectories") && a + 3 < argc)
		{
			trajName = argv[++a];
			trajMode = strcmp(argv[++a], "binary") ? File_Io::ASCII : File_Io::BINARY;
			trajChunk = atoi(argv[++a]);
		}
		else if (!strcmp(argv[a], "--grids") && a + 2 < argc)
		{
			gridName = argv[++a];
			gridMode = strcmp(argv[++a], "binary") ? File_Io::ASCII : File_Io::BINARY;
		}
		else if (!strcmp(argv[a], "--surfaces") && a + 3 < argc)
		{
			surfName = argv[++a];
			surfMode = strcmp(argv[++a], "binary") ? File_Io::ASCII : File_Io::BINARY;
			surfNeighbours = atoi(argv[++a]) != 0;
		}
		else { fprintf(stderr, "unknown option %s\n", argv[a]); return 2; }
	}
	File_Io::LogTrajectory* trajLog = trajName ? new File_Io::LogTrajectory(trajName, trajMode, 0, trajChunk) : 0;
	File_Io::LogGrid* gridLog = 0;  // created once the system is loaded
	File_Io::LogSurface* surfLog = 0;

	std::srand(99); // as main() does (tapsim.cpp:235)

	Process::EvaporationOptions options;
	Process::EvaporationOptions::setDefaults(ini, &options);

	System_3d system;
	system.gridTable.setThreadNum(threads);

	const double tSetup0 = wall_seconds();
	if (dumpIn)
	{
		File_Io::readSystem(dumpIn, &system, 0);
		File_Io::readConfig(cfg, &system.configTable);
		// --no-sync keeps the dump's couplings, as `tapsim resumption` does
		// (tapsim.cpp:195-231); otherwise recompute them (doEvaporation)
		if (!noSync) system.gridTable.fastSync(system.geomTable, system.configTable);
	}
	else
		Process::initialization(cfg, nodes, &system);
	const double tSetup1 = wall_seconds();

	if (!initGiven)
	{
		initThr = options.refreshThreshold;
		initCycle = options.refreshCycleSize;
		initQueue = options.refreshQueueSize;
	}
	const double tRelax0 = wall_seconds();
	if (initRelax) Process::relaxation(initThr, initCycle, initQueue, &system);
	const double tRelax1 = wall_seconds();

	if (phiName)
	{
		FILE* f = fopen(phiName, "wb");
		write_phi(f, system);
		fclose(f);
	}
	FILE* phiEvents = phiEventsName ? fopen(phiEventsName, "wb") : 0;

	std::vector<int> forced;
	if (forceName)
	{
		std::ifstream ff(forceName);
		int v;
		while (ff >> v) forced.push_back(v);
	}

	Surface_3d::Table surfaceTable;
	surfaceTable.setVacuumId(system.configTable[options.vacuumName.c_str()].id());
	surfaceTable.init(system);
	Surface_3d::evap_compute_specificFields(&surfaceTable, system);
	Surface_3d::evap_compute_probabilities(options.probMode, &surfaceTable, system);
	update_coordination(&system);

	FILE* out = fopen(outName, "w");
	fprintf(out, "# setup_s %.6f init_relax_s %.6f nodes %d tets %d surface %d\n",
		tSetup1 - tSetup0, tRelax1 - tRelax0, system.geomTable.numNodes(),
		system.geomTable.numTetrahedra(), (int)surfaceTable.nodes().size());
	fprintf(out, "# event node id prob best second margin phiBefore EbX EbY EbZ phiAfter EaX EaY EaZ "
		"startX startY startZ stopX stopY stopZ time timeScale voltage status npts "
		"lastPhi apexX apexY apexZ nX nY nZ wall_s\n");

	std::queue<float> voltageQueue;
	float voltageQueueSum(0.0f);

	for (int ev = 0; ev < nEvents && surfaceTable.nodes().size() > 0; ev++)
	{
		const double t0 = wall_seconds();
		const float scalingReference = surfaceTable.scalingReference();

		// near-tie bookkeeping: top two probabilities over the surface set
		float best = -1.0f, second = -1.0f;
		for (Surface_3d::Nodeset::const_iterator i = surfaceTable.nodes().begin(); i != surfaceTable.nodes().end(); i++)
		{
			const float p = i->probability();
			if (p > best) { second = best; best = p; }
			else if (p > second) second = p;
		}

		// I) choose
		Surface_3d::Nodeset::const_iterator node = Surface_3d::evap_findCandidate(options.evapMode, surfaceTable);
		int nodeIndex = node->index();
		float probability = node->probability();
		if (ev < (int)forced.size())
		{
			Surface_3d::Nodeset::const_iterator f = surfaceTable.nodes().find(Surface_3d::Node(forced[ev]));
			if (f == surfaceTable.nodes().end()) { fprintf(stderr, "forced node %d not on surface\n", forced[ev]); return 3; }
			nodeIndex = f->index();
			probability = f->probability();
		}
		const int nodeId = system.gridTable.id(nodeIndex).toValue();
		const float potentialBefore = system.gridTable.potential(nodeIndex);
		const MathVector3d<float> fieldBefore = system.gridTable.field_o1(nodeIndex, system.geomTable);
		const Geometry_3d::Point apex = system.geomTable.nodeCoords(surfaceTable.apex(system)->index());
		const Geometry_3d::Point normal = surfaceTable.normal(nodeIndex, system);

		// II) remove
		const Configuration::NodeId removedId = system.gridTable.id(nodeIndex);
		evap_takeAway(&system, &surfaceTable, nodeIndex);
		update_coordination(&system);

		// III) relax
		try { system.gridTable.localRelax(nodeIndex, options.relaxShellSize, options.relaxThreshold, options.relaxCycleSize, options.relaxQueueSize); }
		catch (Grid_3d::Table::RelaxationFault&) {}
		try { system.gridTable.relax(options.relaxGlobalCycles); }
		catch (Grid_3d::Table::RelaxationFault&) {}
		if (options.refreshInterval > 0 && (options.initEventCnt + ev + 1) % options.refreshInterval == 0)
		{
			try { system.gridTable.relax(options.refreshThreshold, options.refreshCycleSize, options.refreshQueueSize); }
			catch (Grid_3d::Table::RelaxationFault&) {}
		}

		// IV) fields and probabilities
		Surface_3d::evap_compute_specificFields(&surfaceTable, system);
		Surface_3d::evap_compute_probabilities(options.probMode, &surfaceTable, system);

		// V) trajectory
		float charge = system.configTable[removedId].evapCharge();
		charge *= Trajectory_3d::eCharge;
		float mass = system.configTable[removedId].mass();
		mass *= Trajectory_3d::amu2kg;
		const Geometry_3d::Point position = system.geomTable.nodeCoords(nodeIndex);
		const MathVector3d<float> velocity(0.0f);

		Trajectory_3d trajectory;
		trajectory.setGeometry(&system.geomTable);
		trajectory.setGrid(&system.gridTable);
		trajectory.setIntegratorType(options.trajectoryIntegrator);
		trajectory.setStepperType(options.trajectoryStepper);
		trajectory.setTimeStepLimit(options.trajectoryTimeStepLimit);
		const int tetGuess = system.geomTable.node(nodeIndex).associatedTetrahedron;
		trajectory.init(position, velocity, charge, mass, tetGuess);
		const int status = trajectory.integrate(options.trajectoryTimeStep, options.trajectoryErrorThreshold);
		trajectory.extrapolate(Geometry_3d::Point::Z, system.geomTable.max().z());

		// VI) voltage and time scale
		const float potentialAfter = system.gridTable.potential(nodeIndex);
		const MathVector3d<float> fieldAfter = system.gridTable.field_o1(nodeIndex, system.geomTable);
		float voltage, timeScale, lastPhi = 0.0f;
		std::vector<Trajectory_3d::phaseVector>::const_reverse_iterator back = trajectory.data().rbegin();
		while (trajectory.data().rend() != back && back->tetIndex() < 0) back++;
		if (trajectory.data().rend() != back && fieldBefore.length() != 0.0f)
		{
			lastPhi = Grid_3d::potential(system.geomTable, system.gridTable, back->position(), back->tetIndex());
			float v = potentialBefore;
			v -= lastPhi;
			v *= system.configTable[removedId].evapField();
			v /= fieldBefore.length();
			v /= scalingReference;
			voltageQueue.push(v);
			voltageQueueSum += v;
			while (voltageQueue.size() > options.voltageQueueSize)
			{
				voltageQueueSum -= voltageQueue.front();
				voltageQueue.pop();
			}
			voltage = voltageQueueSum / voltageQueue.size();
			timeScale = potentialAfter;
			timeScale -= lastPhi;
			timeScale /= voltage;
			timeScale = std::sqrt(timeScale);
		}
		else
		{
			voltage = (fieldBefore.length() == 0.0f) ? 1.0f : 0.0f;
			timeScale = 1.0f;
		}
		const double t1 = wall_seconds();

		const Trajectory_3d::phaseVector& first = trajectory.data().front();
		const Trajectory_3d::phaseVector& last = trajectory.data().back();
		const float margin = best > 0.0f ? (best - second) / best : 0.0f;
		fprintf(out, "%d %d %d %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g "
			"%.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %d %d %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.6f\n",
			ev + 1, nodeIndex, nodeId, probability, best, second, margin,
			potentialBefore, fieldBefore[0], fieldBefore[1], fieldBefore[2],
			potentialAfter, fieldAfter[0], fieldAfter[1], fieldAfter[2],
			first.position()[0], first.position()[1], first.position()[2],
			last.position()[0], last.position()[1], last.position()[2],
			last.time(), timeScale, voltage, status, (int)trajectory.data().size(),
			lastPhi, apex[0], apex[1], apex[2], normal[0], normal[1], normal[2], t1 - t0);
		fflush(out);
		if (phiEvents) write_phi(phiEvents, system);
		if (trajLog) trajLog->push(ev + 1, system.gridTable.number(nodeIndex).toValue(), timeScale, trajectory);
		if (gridName)
		{
			if (!gridLog) gridLog = new File_Io::LogGrid(gridName, &system.geomTable, &system.configTable, gridMode);
			gridLog->push(ev + 1, system.gridTable);
		}
		if (surfName)
		{
			if (!surfLog) surfLog = new File_Io::LogSurface(surfName, &system, surfMode, 0, 0, surfNeighbours);
			surfLog->push(ev + 1, surfaceTable);
		}
	}
	// the destructors join the writer threads after they have written their queues
	delete trajLog;
	delete gridLog;
	delete surfLog;
	fclose(out);
	if (phiEvents) fclose(phiEvents);
	return 0;
}

// ref_harness face <dump> <n1> <n2> ... : Voronoi face of each pair as the
// reference computes it (get_voronoiFace + finiteArea with the coupling's
// infinity factor 0.5*d and the surface test's factor 1.0).
static int cmd_face(int argc, char** argv)
{
	System_3d system;
	system.gridTable.setThreadNum(1);
	File_Io::readSystem(argv[2], &system, 0);
	for (int a = 3; a + 1 < argc; a += 2)
	{
		const int n1 = atoi(argv[a]), n2 = atoi(argv[a + 1]);
		Geometry_3d::VoronoiFace face;
		system.geomTable.get_voronoiFace(n1, n2, &face);
		const float d = system.geomTable.distance(n1, n2);
		printf("pair %d %d finite %d ntets %d areaHalf %.9g areaOne %.9g d %.9g\n", n1, n2, (int)face.isFinite(),
			(int)face.tets.size(), face.finiteArea(0.5f * d), face.finiteArea(1.0f), d);
		for (std::list<Geometry_3d::Point>::const_iterator v = face.vertices.begin(); v != face.vertices.end(); v++)
			printf("  v %.9g %.9g %.9g\n", (*v)[0], (*v)[1], (*v)[2]);
	}
	return 0;
}

int main(int argc, char** argv)
{
	if (argc < 2) { fprintf(stderr, "usage: ref_harness mesh|evap ...\n"); return 2; }
	try
	{
		if (!strcmp(argv[1], "mesh")) return cmd_mesh(argc, argv);
		if (!strcmp(argv[1], "evap")) return cmd_evap(argc, argv);
		if (!strcmp(argv[1], "face")) return cmd_face(argc, argv);
	}
	catch (std::exception& e)
	{
		fprintf(stderr, "ref_harness: %s\n", e.what());
		return 1;
	}
	fprintf(stderr, "unknown command %s\n", argv[1]);
	return 2;
}
